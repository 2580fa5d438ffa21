#!/usr/bin/env python
"""Benchmark of the CSR analytics path on B200.

Workload (one "step"): BFS from each of 64 seeded random non-isolated
sources on an undirected RMAT graph, scale 24, edge factor 16, seed 7,
a/b/c/d = .57/.19/.19/.05, permuted ids, duplicates and self-loops removed
(16.8 M vertices, ~0.5 G CSR entries; ~2.1 GB of col, larger than the
126 MB L2, so no L2 flush is needed between steps).

  value  GTEPS = sum over sources of m_r (CSR entries out of reached
         vertices) / device time, inputs resident in HBM
  e2e    the same metric through the C ABI with the depth vector of every
         BFS copied to pinned host memory inside the timed region (the
         reference's Cuda_BFS returns a host vector too)

Also measured (in "extra"): SSSP GTEPS, PageRank GB/s (FP32+Kahan, FP64),
WCC / CDLP / TC times, the 64-source bitmask BFS, and the 4096x4096 grid.

--impl reference times the reference's own CPU BFS (oracle/_ref, compiled
from the reference's sources) on the same graph, built on the host.
Under torchrun every rank runs its own sources on its own copy of the graph
(replicas, weak scaling; no collective on the data path).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "GTEPS BFS/SSSP, PR GB/s vs HBM peak; learned+batched vs plain, 1x B200"
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--scale", type=int, default=24)
    ap.add_argument("--edge-factor", type=int, default=16)
    ap.add_argument("--seed", type=int, default=7)
    ap.add_argument("--sources", type=int, default=64)
    ap.add_argument("--extras", type=int, default=1, help="also measure the other algorithms")
    ap.add_argument("--cpu-sample", type=int, default=1, help="number of BFS sources in the CPU baseline")
    ap.add_argument("--parity", type=int, default=1,
                    help="check the outputs at the benchmark sizes against the CPU checkers and time the "
                         "reference's CPU code for all six algorithms (rank 0, outside the timed regions)")
    ap.add_argument("--only", default=None,
                    choices=["bfs", "sssp", "wcc", "pr", "pr64", "cdlp", "tc", "msbfs64", "msbfs256", "mssssp256", "gpma"],
                    help="profiling driver: run one algorithm --warmup + --steps times on the RMAT graph of "
                         "--scale and print its mean time (not a bench line)")
    ap.add_argument("--gpma-sizes", default="1000,100000,10000000",
                    help="update batch sizes of the dynamic-graph section (--only gpma)")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def profiled_traffic(args):
    """DRAM bytes (read + write) per BFS launch from the committed ncu summary
    of this workload (RMAT scale 24, edge factor 16, seed 7), else None."""
    if (args.scale, args.edge_factor, args.seed) != (24, 16, 7):
        return None
    path = os.path.join(ROOT, "profiles", "bfs_persistent_kernel_rmat24_dram.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1])
    except OSError:
        pass
    return None


def pick_sources(rowptr_host: np.ndarray, count: int, seed: int, salt: int = 0):
    """Seeded random non-isolated sources (splitmix64 draws, first hits)."""
    n = len(rowptr_host) - 1
    deg = np.diff(rowptr_host)
    out = []
    k = 0
    mask = (1 << 64) - 1

    def mix(z):
        z = (z + 0x9E3779B97F4A7C15) & mask
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & mask
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & mask
        return z ^ (z >> 31)

    base = mix(seed * 1000003 + 5 + salt * 7919)
    while len(out) < count and k < 100 * count + 1000:
        v = mix(base ^ k) % n
        k += 1
        if deg[v] > 0:
            out.append(int(v))
    return out


class ClockSampler:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "100"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        if args.impl == "ours":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
        else:
            dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=1800))
    return world, rank, local


def barrier_sync(world):
    import torch
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    if torch.cuda.is_available():
        torch.cuda.synchronize()


def reduce_over_ranks(world, x: float, op: str = "max") -> float:
    """max or sum of a per-rank number over all ranks (a host-side scalar;
    CPU tensors under gloo, device tensors under NCCL)."""
    if world <= 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
    return float(t.item())


def max_over_ranks(world, x: float) -> float:
    return reduce_over_ranks(world, x, "max")


def replica_gteps(world, edges_this_rank: int, ms_this_rank: float):
    """Whole-job GTEPS of independent replicas: the entries every rank
    reached, over the slowest rank's device time."""
    total = reduce_over_ranks(world, float(edges_this_rank), "sum")
    ms = reduce_over_ranks(world, ms_this_rank, "max")
    return total / (ms / 1e3) / 1e9, total, ms


# ---------------------------------------------------------------- ours
def run_ours(args, world, rank, local):
    import ctypes

    import torch

    import graphhet_b200 as G

    torch.cuda.set_device(local)
    # A non-default stream: the legacy default stream would serialise the
    # e2e copy stream against every kernel.
    work_stream = torch.cuda.Stream()
    torch.cuda.set_stream(work_stream)
    ws = G.default_workspace()
    t0 = time.time()
    g = G.rmat_graph(args.scale, args.edge_factor, args.seed, directed=False)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    # One-time preparation (the reference's toCSR step): degree relabelling.
    rg = G.ResidentGraph(g)
    torch.cuda.synchronize()
    n, m = g.n, g.m
    rp_host = g.rowptr.cpu().numpy()
    srcs = pick_sources(rp_host, args.sources, args.seed, salt=rank)
    depth = torch.empty(n, dtype=torch.int32, device="cuda")
    L = G.lib()
    wsh = ws.handle
    opt_plain = G.BfsOptions(policy=G.POLICY_HEURISTIC)
    trace_cap = 64
    trace = (ctypes.c_float * (trace_cap * G.TRACE_COLS))()
    opt_trace = G.BfsOptions(policy=G.POLICY_HEURISTIC, record_trace=1, trace=ctypes.cast(trace, ctypes.c_void_p),
                             trace_cap=trace_cap)
    st = G.TraversalStats()
    rp_p, col_p, d_p = G._ptr(g.rowptr), G._ptr(g.col), G._ptr(depth)

    def one_bfs(s, opt):
        G._check(L.ghb_graph_bfs(wsh, rg._h, s, G.INT32_MAX, d_p, ctypes.byref(opt), ctypes.byref(st)),
                 "ghb_graph_bfs")
        return st.edges_reached

    def one_bfs_raw(s, opt):
        G._check(L.ghb_bfs(wsh, n, rp_p, col_p, rp_p, col_p, s, G.INT32_MAX, d_p, ctypes.byref(opt),
                           ctypes.byref(st)), "ghb_bfs")
        return st.edges_reached

    # m_r per source (deterministic) and warm-up.
    mr = {}
    for s in srcs:
        mr[s] = one_bfs(s, opt_plain)
    for _ in range(max(0, args.warmup - 1)):
        for s in srcs:
            one_bfs(s, opt_plain)
    l0, _ = ws.counters()

    # ---- timed region: K steps, every step = BFS from every source.  Each
    # BFS is one cooperative launch (bfs_persistent_kernel); the library times
    # each launch with CUDA events on this stream (stats.device_ms).
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launch_ms = []
    with ClockSampler(local) as clk:
        barrier_sync(world)
        torch.cuda.nvtx.range_push("timed")
        ev0.record(stream)
        for _ in range(args.steps):
            for s in srcs:
                one_bfs(s, opt_plain)
                launch_ms.append(st.device_ms)
        ev1.record(stream)
        torch.cuda.nvtx.range_pop()
        barrier_sync(world)
    l1, _ = ws.counters()
    edges_per_step = sum(mr[s] for s in srcs)
    value, total_edges, ms = replica_gteps(world, edges_per_step * args.steps, ev0.elapsed_time(ev1))
    launches = int(l1 - l0)

    # ---- roofline of the dominant kernel (the whole-traversal BFS launch):
    # algorithmic bytes per launch = 4(n+1) + 4 m_r + 4 n (rowptr, the entries
    # out of reached vertices, depth), over that launch's event time.
    hbm, peak_kind = measured_peaks()
    bytes_per = [4 * (n + 1) + 4 * mr[s] + 4 * n for _ in range(args.steps) for s in srcs]
    achieved = sum(bytes_per) / (sum(launch_ms) / 1e3) / 1e9
    roofline = {"bound": "hbm", "kernel": "bfs_persistent_kernel", "achieved": round(achieved, 1), "peak": hbm,
                "unit": "GB/s", "frac": round(achieved / hbm, 4), "peak_source": peak_kind, "traffic": profiled_traffic(args),
                "traffic_source": "profiles/bfs_persistent_kernel_rmat24_dram.md (ncu, 3 launches)",
                "bytes_per_launch": int(sum(bytes_per) / len(bytes_per)),
                "launch_ms_mean": round(sum(launch_ms) / len(launch_ms), 4), "launches": len(launch_ms),
                "share_of_step": round(sum(launch_ms) / ms, 3) if world == 1 else None}

    # ---- e2e: through the C ABI, every depth vector copied to pinned host
    # memory inside the timed region.  The copy of one source's result runs on
    # a second stream while the next source's BFS computes (two device and
    # two pinned host buffers, ordered by events).
    dbuf = [depth, torch.empty(n, dtype=torch.int32, device="cuda")]
    hbuf = [torch.empty(n, dtype=torch.int32, pin_memory=True) for _ in range(2)]
    copy_stream = torch.cuda.Stream()
    done_bfs = [torch.cuda.Event(), torch.cuda.Event()]
    done_copy = [torch.cuda.Event(), torch.cuda.Event()]
    barrier_sync(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    i = 0
    for _ in range(args.steps):
        for s in srcs:
            k = i & 1
            stream.wait_event(done_copy[k])  # the copy of result i-2 has left dbuf[k]
            G._check(L.ghb_graph_bfs(wsh, rg._h, s, G.INT32_MAX, G._ptr(dbuf[k]), ctypes.byref(opt_plain),
                                     ctypes.byref(st)), "ghb_graph_bfs")
            done_bfs[k].record(stream)
            with torch.cuda.stream(copy_stream):
                copy_stream.wait_event(done_bfs[k])
                hbuf[k].copy_(dbuf[k], non_blocking=True)
                done_copy[k].record(copy_stream)
            i += 1
    stream.wait_stream(copy_stream)
    e1.record(stream)
    barrier_sync(world)
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1))
    e2e_int32 = {"value": round(total_edges / (e2e_ms / 1e3) / 1e9, 3), "unit": "GTEPS",
                 "d2h_bytes_per_step": 4 * n * len(srcs),
                 "note": "ghb_graph_bfs into a device buffer, then a torch copy of the int32 depths to pinned host "
                         "memory on a second stream, overlapped with the next BFS"}
    del dbuf, hbuf

    # ---- e2e through the C ABI's host-buffer entry: every step is one
    # ghb_graph_bfs_many_host call that leaves all 64 depth vectors, int32,
    # in a host array (traversal, byte copy over PCIe and host widening
    # pipelined inside the call).  The array is written once before timing
    # so that no page is first touched inside the timed region.
    host_out = np.zeros((len(srcs), n), dtype=np.int32)
    rg.bfs_many_host(srcs, out=host_out)
    barrier_sync(world)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        _, hst = rg.bfs_many_host(srcs, out=host_out)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier_sync(world)
    e2e_ms = max_over_ranks(world, e0.elapsed_time(e1))
    byte_rows = hst["levels"] < 255
    e2e = {"value": round(total_edges / (e2e_ms / 1e3) / 1e9, 3), "unit": "GTEPS",
           "h2d_bytes_per_step": 4 * len(srcs), "d2h_bytes_per_step": (1 if byte_rows else 4) * n * len(srcs),
           "note": "ghb_graph_bfs_many_host: all 64 depth vectors as int32 in a host array each step; the GPU "
                   "traverses one source while the copy engine brings the previous one's depths as one byte "
                   "each and host threads widen the one before",
           "int32_copy_variant": e2e_int32}
    del host_out

    out = {
        "metric": METRIC, "value": round(value, 3), "unit": "GTEPS", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        "config": {"workload": f"BFS from {len(srcs)} random non-isolated sources, undirected RMAT "
                               f"scale {args.scale} edge factor {args.edge_factor} seed {args.seed}",
                   "n": n, "m": m, "sources_per_step": len(srcs),
                   "l2": "inputs larger than L2 (col %.2f GB)" % (4 * m / 1e9),
                   "parallelism": f"replicas x{world}"},
        "policy": "heuristic (alpha 256, beta 24)",
        "roofline": roofline, "e2e": e2e, "gpu_launches": launches, "build_s": round(build_s, 2),
        "relabel_ms": round(rg.build_ms, 1), "n_active": rg.n_active,
    }
    # The same sources on the caller's CSR without the relabelled handle.
    torch.cuda.synchronize()
    r0, r1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    r0.record(stream)
    for s in srcs:
        one_bfs_raw(s, opt_plain)
    r1.record(stream)
    torch.cuda.synchronize()
    out["raw_csr_bfs_gteps"] = round(edges_per_step / (r0.elapsed_time(r1) / 1e3) / 1e9, 3)
    out["clocks"] = clk.summary()

    parity = {}
    if rank == 0 and args.extras:
        out["extra"] = extras(args, G, g, rg, srcs, ws, parity if args.parity else None)
        out["dropin_e2e"] = dropin_leg(args, srcs[:8])
    if rank == 0 and args.parity:
        # Outputs at the benchmark size against the CPU checkers, and the
        # reference's CPU code timed on the same graph (outside every timed
        # region above).
        cpu = cpu_section(args, G, g, rg, srcs, parity, dict(out.get("extra", {}), bfs_gteps_single=out["value"]))
        out.setdefault("extra", {})["parity"] = parity
        out["cpu_baselines"] = cpu
        if "bfs" in cpu:
            b = cpu["bfs"]
            out["cpu_baseline"] = {"value": b["cpu"], "unit": "GTEPS", "cores": b["cores"], "kind": b["kind"],
                                   "sample": b["sample"]}
    elif rank == 0 and args.cpu_sample > 0:
        out["cpu_baseline"] = cpu_baseline_port(g, srcs[: args.cpu_sample])
    return out


def timed(fn, reps=1):
    import torch
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    s.record()
    r = None
    for _ in range(reps):
        r = fn()
    e.record()
    torch.cuda.synchronize()
    return s.elapsed_time(e) / reps, r


def extras(args, G, g, rg, srcs, ws, parity=None):
    import torch
    hbm, _ = measured_peaks()
    n, m = g.n, g.m
    ex = {}
    # SSSP over 4 sources
    dist = torch.empty(n, dtype=torch.float64, device="cuda")
    rg.sssp(srcs[0], out=dist)
    t_tot, e_tot = 0.0, 0
    for s in srcs[:4]:
        ms, (d, st) = timed(lambda: rg.sssp(s, out=dist))
        t_tot += ms
        e_tot += st["edges_reached"]
    ex["sssp_gteps"] = round(e_tot / (t_tot / 1e3) / 1e9, 3)
    ex["sssp_ms_per_source"] = round(t_tot / 4, 3)
    # PageRank: 10 iterations, FP32+Kahan and FP64
    rank = torch.empty(n, dtype=torch.float64, device="cuda")
    for prec, name, vb in ((G.PR_FP32_KAHAN, "fp32_kahan", 8), (G.PR_FP64, "fp64", 16)):
        rg.pagerank(10, 0.85, precision=prec, out=rank)
        ms, _ = timed(lambda: rg.pagerank(10, 0.85, precision=prec, out=rank), reps=2)
        per_it = ms / 10
        bytes_it = 4 * (n + 1) + 4 * m + vb * n
        ex[f"pr_{name}_ms_per_iter"] = round(per_it, 4)
        ex[f"pr_{name}_gbs"] = round(bytes_it / (per_it / 1e3) / 1e9, 1)
        ex[f"pr_{name}_frac_hbm"] = round(bytes_it / (per_it / 1e3) / 1e9 / hbm, 4)
    lab = torch.empty(n, dtype=torch.int32, device="cuda")
    rg.wcc(out=lab)
    ms, _ = timed(lambda: rg.wcc(out=lab), reps=3)
    ex["wcc_ms"] = round(ms, 3)
    ex["wcc_gbs"] = round((4 * (n + 1) + 4 * m + 4 * n) / (ms / 1e3) / 1e9, 1)
    rg.cdlp(10, out=lab)
    ms, _ = timed(lambda: rg.cdlp(10, out=lab))
    ex["cdlp_ms_per_iter"] = round(ms / 10, 3)
    ex["cdlp_gbs"] = round((4 * (n + 1) + 4 * m + 8 * n) / (ms / 10 / 1e3) / 1e9, 1)
    # The first call on a graph also checks the input (symmetric, sorted,
    # loop-free) and keeps the result on the graph; timed apart.
    ms0, _ = timed(lambda: rg.tc())
    ex["tc_first_call_ms"] = round(ms0, 2)
    ms, (c64, c32, tri) = timed(lambda: rg.tc())
    ex["tc_ms"] = round(ms, 2)
    ex["tc_triangles"] = int(tri)
    ex["tc_edges_per_s"] = round(m / (ms / 1e3) / 1e9, 3)
    # 64-source bitmask BFS vs 64 single-source runs
    import ctypes
    k = min(64, len(srcs))
    sd = torch.tensor(srcs[:k], dtype=torch.int32, device="cuda")
    out = torch.empty(k * n, dtype=torch.int32, device="cuda")
    stt = G.TraversalStats()

    def ms_bfs():
        G._check(G.lib().ghb_graph_msbfs(ws.handle, rg._h, G._ptr(sd), k, G._ptr(out), ctypes.byref(stt)),
                 "ghb_graph_msbfs")
    ms_bfs()
    ms, _ = timed(ms_bfs)
    mr_sum = 0
    for s in srcs[:k]:
        mr_sum += rg.bfs(s, out=lab)[1]["edges_reached"]
    ex["msbfs64_ms"] = round(ms, 2)
    ex["msbfs64_gteps"] = round(mr_sum / (ms / 1e3) / 1e9, 3)
    del out
    torch.cuda.empty_cache()
    # Learned schedule policy (trained on the 400-graph family; this graph is
    # held out): GTEPS over the same sources, and regret of each policy
    # against the replayed per-level oracle schedule.
    from graphhet_b200 import policy as P
    if os.path.exists(P.WEIGHTS_PATH):
        P.install()

        def bfs_sum(**kw):
            t = 0.0
            for s in srcs:
                t += rg.bfs(s, out=lab, **kw)[1]["device_ms"]
            return t
        bfs_sum(policy=G.POLICY_LEARNED)
        t_h, t_l = bfs_sum(policy=G.POLICY_HEURISTIC), bfs_sum(policy=G.POLICY_LEARNED)
        ex["learned_bfs_gteps"] = round(mr_sum / (t_l / 1e3) / 1e9, 3)
        ex["heuristic_bfs_gteps_same_run"] = round(mr_sum / (t_h / 1e3) / 1e9, 3)
        r = P.regret(rg, srcs[:8])
        ex["regret_rmat"] = {k: (round(v, 4) if isinstance(v, float) else {a: round(b, 3) for a, b in v.items()})
                             for k, v in r.items()}
        t_rule = t_net = 0.0
        for s in srcs[:4]:
            t_rule += rg.sssp(s, out=dist)[1]["device_ms"]
            t_net += rg.sssp(s, out=dist, policy=G.POLICY_LEARNED)[1]["device_ms"]
        ex["sssp_learned_ms_per_source"] = round(t_net / 4, 3)
        ex["sssp_rule_ms_per_source"] = round(t_rule / 4, 3)
        ex["learned_vs_plain"] = round(t_h / t_l, 3)
        ex["batched_vs_plain"] = round((mr_sum / (ms / 1e3)) / (mr_sum / (t_h / 1e3)), 3)
    # PageRank precision: RMAT seed 11 scale 25 directed with ~10 % of the
    # vertices dangling; FP32 ranks + Kahan rows (FP64 sink mass and L1)
    # against the FP64 path, per iteration, and run to L1 change 1e-9.
    del rank, lab
    torch.cuda.empty_cache()
    ex["pr_precision"] = pr_precision(G, hbm, parity=parity)
    torch.cuda.empty_cache()
    # Batched sources (RMAT seed 3 scale 22, 256 sources): one 256-source
    # pass (4 words per vertex) against 256 single-source traversals.
    g22 = G.rmat_graph(22, 16, 3)
    bsrc = pick_sources(g22.rowptr.cpu().numpy(), 256, 3)
    gb = G.ResidentGraph(g22)
    del g22
    lb = torch.empty(gb.n, dtype=torch.int32, device="cuda")
    mr_b, t_single = 0, 0.0
    for s in bsrc:
        gb.bfs(s, out=lb)
    for s in bsrc:
        _, stb = gb.bfs(s, out=lb)
        mr_b += stb["edges_reached"]
        t_single += stb["device_ms"]
    ob = torch.empty(256 * gb.n, dtype=torch.int32, device="cuda")
    gb.msbfs(bsrc, out=ob)
    ms256, _ = timed(lambda: gb.msbfs(bsrc, out=ob))
    ms64, _ = timed(lambda: gb.msbfs(bsrc[:64], out=ob))
    mr_64 = 0
    for s in bsrc[:64]:
        mr_64 += gb.bfs(s, out=lb)[1]["edges_reached"]
    ex["batch256_rmat22_single_gteps"] = round(mr_b / (t_single / 1e3) / 1e9, 3)
    ex["batch256_rmat22_msbfs_ms"] = round(ms256, 2)
    ex["batch256_rmat22_msbfs_gteps"] = round(mr_b / (ms256 / 1e3) / 1e9, 3)
    ex["batch64_rmat22_msbfs_gteps"] = round(mr_64 / (ms64 / 1e3) / 1e9, 3)
    ex["batch256_vs_plain"] = round(t_single / ms256, 3)
    # The 256-source pass's directions: the rule and the learned model
    # against the per-level oracle (levels timed pushed and pulled).
    from graphhet_b200 import policy as P
    if os.path.exists(P.MS_WEIGHTS_PATH):
        P.ms_install()
        r = P.ms_regret(gb, bsrc, learned=True)
        ex["regret_msbfs256_rmat22"] = {"ms": {a: round(b, 3) for a, b in r["ms"].items()},
                                        "regret_rule": round(r["regret_rule"], 4),
                                        "regret_learned": round(r["regret_learned"], 4),
                                        "rule_dirs": r["rule_dirs"], "learned_dirs": r["learned_dirs"],
                                        "oracle_dirs": r["oracle_dirs"]}
    del ob
    # 256 SSSP sources on the same graph: one bucketed multi-source pass
    # against 256 single-source runs (weight rule's width in both).
    dsum = torch.empty(gb.n, dtype=torch.float64, device="cuda")
    er_s, t_s = 0, 0.0
    for s in bsrc:
        _, sts = gb.sssp(s, out=dsum)
        er_s += sts["edges_reached"]
        t_s += sts["device_ms"]
    dms = torch.empty(256 * gb.n, dtype=torch.float64, device="cuda")
    gb.mssssp(bsrc, out=dms)
    ms_sp, _ = timed(lambda: gb.mssssp(bsrc, out=dms))
    same = all(torch.equal(dms.view(256, gb.n)[i], gb.sssp(bsrc[i], out=dsum)[0]) for i in (0, 101, 255))
    ex["batch256_sssp_single_ms"] = round(t_s, 1)
    ex["batch256_sssp_single_gteps"] = round(er_s / (t_s / 1e3) / 1e9, 3)
    ex["batch256_sssp_ms"] = round(ms_sp, 1)
    ex["batch256_sssp_gteps"] = round(er_s / (ms_sp / 1e3) / 1e9, 3)
    ex["batch256_sssp_vs_plain"] = round(t_s / ms_sp, 3)
    ex["batch256_sssp_identical"] = bool(same)
    del dms, dsum, gb
    torch.cuda.empty_cache()
    # Many small graphs (2,000 ER graphs, n log-uniform in [1k, 200k], mean
    # degree uniform in [2, 32], seed 5) as one disjoint-union CSR: WCC + TC
    # of all of them in one launch-only call, eager and replayed from a CUDA
    # graph, against the per-graph entry points.
    ex["batch_er2000"] = er_batch_section(G, ws)
    torch.cuda.empty_cache()
    # Dynamic graph: batched edge updates on this RMAT graph.
    ex["gpma_rmat"] = gpma_section(G, g)
    torch.cuda.empty_cache()
    # 4096 x 4096 grid: BFS and SSSP from its centre
    grid = G.grid_graph(4096, 4096, weight_seed=args.seed)
    gg = G.ResidentGraph(grid)
    c = 2048 * 4096 + 2048
    dg = torch.empty(gg.n, dtype=torch.int32, device="cuda")
    gg.bfs(c, out=dg)
    ms, (_, st) = timed(lambda: gg.bfs(c, out=dg))
    ex["grid_bfs_ms"] = round(ms, 2)
    ex["grid_bfs_levels"] = st["levels"]
    ex["grid_bfs_gteps"] = round(st["edges_reached"] / (ms / 1e3) / 1e9, 3)
    dgs = torch.empty(gg.n, dtype=torch.float64, device="cuda")
    gg.sssp(c, out=dgs)  # warm-up: scratch and the light ends of this width
    ms, (_, st) = timed(lambda: gg.sssp(c, out=dgs))
    ex["grid_sssp_ms"] = round(ms, 2)
    ex["grid_sssp_gteps"] = round(st["edges_reached"] / (ms / 1e3) / 1e9, 3)
    if parity is not None:
        parity["grid4096"] = grid_parity(grid, c, dg, dgs)
    del grid
    if G.policy_loaded():
        gg.bfs(c, out=dg, policy=G.POLICY_LEARNED)
        ms, _ = timed(lambda: gg.bfs(c, out=dg, policy=G.POLICY_LEARNED))
        ex["grid_learned_bfs_ms"] = round(ms, 2)
        gg.sssp(c, out=dgs, policy=G.POLICY_LEARNED)  # warm-up: the light ends of the network's width
        ms, _ = timed(lambda: gg.sssp(c, out=dgs, policy=G.POLICY_LEARNED))
        ex["grid_learned_sssp_ms"] = round(ms, 2)
        r = P.regret(gg, [c], repeats=1)
        ex["regret_grid"] = {k: (round(v, 4) if isinstance(v, float) else {a: round(b, 3) for a, b in v.items()})
                             for k, v in r.items()}
    return ex


def gpma_batch(g, size, gen):
    """One mixed update batch on the device: half inserts of random (mostly
    new) edges with weights in (0.25, 2), a quarter deletes of present edges,
    a quarter weight changes of present edges."""
    import torch
    n, m = g.n, g.m
    q = size // 4
    k_new = size - 2 * q
    src = torch.randint(0, n, (k_new,), device="cuda", generator=gen)
    dst = torch.randint(0, n, (k_new,), device="cuda", generator=gen)
    j = torch.randint(0, m, (2 * q,), device="cuda", generator=gen)
    rows = torch.searchsorted(g.rowptr, j.to(torch.int32), right=True) - 1
    keys = torch.cat([(src.to(torch.int64) << 32) | dst, (rows.to(torch.int64) << 32) | g.col[j].to(torch.int64)])
    vals = torch.rand(size, device="cuda", dtype=torch.float64, generator=gen) * 1.75 + 0.25
    vals[k_new: k_new + q] = 0.0
    perm = torch.randperm(size, device="cuda", generator=gen)
    return keys[perm].contiguous(), vals[perm].contiguous()


def gpma_section(G, g, sizes=(1000, 100000, 10000000), reps=(20, 10, 3), seed=7):
    """Dynamic graph (the reference's GPMA update path) on graph g: load from
    its CSR, batches of mixed updates (1,000 is the reference LDBC driver's
    batch, LDBC_GPU_gpma.cu:124-140), each timed with CUDA events around the
    call (which returns after its kernels are queued behind one host sync),
    then the compact-CSR rebuild a following analytic pays, and one BFS on it."""
    import ctypes

    import torch
    out = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dg = G.DynamicGraph.from_csr(g.rowptr, g.col, g.w)
    torch.cuda.synchronize()
    out["load_ms"] = round((time.perf_counter() - t0) * 1e3, 2)
    ms, _ = timed(lambda: dg.csr_view(weights=False))
    out["csr_rebuild_fresh_ms"] = round(ms, 3)
    gen = torch.Generator(device="cuda")
    gen.manual_seed(seed)
    for size, r in zip(sizes, reps):
        batches = [gpma_batch(g, size, gen) for _ in range(r + 1)]
        dg.update(*batches[0])
        times = []
        for k, v in batches[1:]:
            ms, _ = timed(lambda: dg.update(k, v))
            times.append(ms)
        med = statistics.median(times)
        out[f"batch{size}_ms"] = round(med, 4)
        out[f"batch{size}_mupdates_per_s"] = round(size / (med / 1e3) / 1e6, 3)
        del batches
    k, v = gpma_batch(g, 1000, gen)
    dg.update(k, v)
    ms, _ = timed(lambda: dg.csr_view(weights=False))
    out["csr_rebuild_ms"] = round(ms, 3)
    nm = dg.m
    out["csr_rebuild_gbs"] = round((8 * nm + 16 * g.n) / (ms / 1e3) / 1e9, 1)
    dg.csr_view(weights=True)  # the first weighted view allocates its arrays
    dg.update(*gpma_batch(g, 1000, gen))
    ms, _ = timed(lambda: dg.csr_view(weights=True))
    out["csr_rebuild_weights_ms"] = round(ms, 3)
    rp, col, _ = dg.csr_view(weights=False)
    depth = torch.empty(g.n, dtype=torch.int32, device="cuda")
    src = int(torch.argmax(g.rowptr[1:] - g.rowptr[:-1]))
    # undirected: the snapshot is its own in-CSR, so bottom-up levels run too
    call = lambda: G._check(G.lib().ghb_bfs(None, g.n, ctypes.c_void_p(rp), ctypes.c_void_p(col), ctypes.c_void_p(rp),
                                            ctypes.c_void_p(col), src, 2**31 - 1, G._ptr(depth), None, None),
                            "ghb_bfs")
    call()
    ms, _ = timed(call)
    out["bfs_on_snapshot_ms"] = round(ms, 3)
    st = dg.stats()
    out["stats"] = {k: st[k] for k in ("rows_moved", "repacks", "slots_used", "slots")}
    out["m_after"] = nm
    dg.close()
    return out


def er_batch_section(G, ws, n_graphs=2000, seed=5):
    import ctypes

    import torch
    t0 = time.time()
    b = G.er_batch(n_graphs, seed)
    torch.cuda.synchronize()
    build_s = time.time() - t0
    N, m = b.g.n, b.g.m
    b.reserve(ws)
    lab = torch.empty(N, dtype=torch.int32, device="cuda")
    c64 = torch.empty(N, dtype=torch.int64, device="cuda")
    tri = torch.empty(n_graphs, dtype=torch.int64, device="cuda")
    b.wcc_tc(lab, c64, tri, ws=ws)
    eager_ms, _ = timed(lambda: b.wcc_tc(lab, c64, tri, ws=ws), reps=3)
    side = torch.cuda.Stream()
    side.wait_stream(torch.cuda.current_stream())
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.stream(side):
        with torch.cuda.graph(graph, stream=side):
            b.wcc_tc(lab, c64, tri, ws=ws)
    graph.replay()
    torch.cuda.synchronize()
    graph_ms, _ = timed(lambda: graph.replay(), reps=3)
    lab_u, tri_u = lab.clone(), tri.clone()
    del graph
    # Per-graph entry points (ghb_wcc, ghb_tc) on the same union arrays.
    vb = b.vbase_host
    rp_h = b.g.rowptr.cpu().numpy()
    lab1 = torch.empty(N, dtype=torch.int32, device="cuda")
    tot = ctypes.c_int64()
    L = G.lib()
    wsh = ws.handle

    def per_graph():
        tris = []
        for g in range(n_graphs):
            lo, hi = int(vb[g]), int(vb[g + 1])
            rp_l = b.g.rowptr[lo:hi + 1] - int(rp_h[lo])
            col_l = b.g.col[int(rp_h[lo]):int(rp_h[hi])] - lo
            G._check(L.ghb_wcc(wsh, hi - lo, G._ptr(rp_l), G._ptr(col_l), G._ptr(lab1[lo:hi])), "ghb_wcc")
            G._check(L.ghb_tc(wsh, hi - lo, G._ptr(rp_l), G._ptr(col_l), None, None, ctypes.byref(tot)), "ghb_tc")
            tris.append(tot.value)
        return tris
    per_ms, tris = timed(per_graph)
    same = bool(torch.equal(lab1, lab_u)) and tris == tri_u.cpu().tolist()
    return {"workload": f"{n_graphs} Erdos-Renyi graphs, n log-uniform [1k, 200k], mean degree U[2, 32], seed {seed}",
            "n_total": N, "m_total": m, "build_s": round(build_s, 2), "union_eager_ms": round(eager_ms, 2),
            "union_cuda_graph_ms": round(graph_ms, 2), "per_graph_calls_ms": round(per_ms, 1),
            "speedup_vs_per_graph": round(per_ms / graph_ms, 2), "identical_to_per_graph": same,
            "edges_per_s_union": round(m / (graph_ms / 1e3) / 1e9, 3)}


def pr_precision(G, hbm, scale=25, seed=11, fraction=0.1, parity=None):
    import torch
    gp = G.rmat_dangling_graph(scale, 16, seed, fraction)
    n, m = gp.n, gp.m
    outdeg = gp.rowptr[1:] - gp.rowptr[:-1]
    indeg = torch.bincount(gp.col.long(), minlength=n)
    sinks = int(((outdeg == 0) & (indeg > 0)).sum())
    touched = int(((outdeg > 0) | (indeg > 0)).sum())
    rp = G.ResidentGraph(gp)
    host_in = None
    if parity is not None:
        irp, icol, _ = gp.in_csr()
        host_in = (irp.cpu().numpy(), icol.cpu().numpy(), gp.rowptr.cpu().numpy())
        del irp, icol
    del gp, outdeg, indeg
    torch.cuda.empty_cache()
    r32 = torch.empty(n, dtype=torch.float64, device="cuda")
    r64 = torch.empty(n, dtype=torch.float64, device="cuda")
    rel, mx = [], []
    for it in range(1, 21):
        rp.pagerank(it, 0.85, precision=G.PR_FP32_KAHAN, out=r32)
        rp.pagerank(it, 0.85, precision=G.PR_FP64, out=r64)
        d = (r32 - r64).abs()
        rel.append(float(d.sum() / r64.abs().sum()))
        mx.append(float(d.max()))
    out = {"workload": f"RMAT scale {scale} edge factor 16 seed {seed}, directed, out-edges of ~{fraction:.0%} of "
                       f"the vertices dropped", "n": n, "m": m, "sinks_with_in_edges": sinks,
           "vertices_with_edges": touched}
    bytes_it = {"fp32_kahan": 4 * (n + 1) + 4 * m + 8 * n, "fp64": 4 * (n + 1) + 4 * m + 16 * n}
    for prec, name in ((G.PR_FP32_KAHAN, "fp32_kahan"), (G.PR_FP64, "fp64")):
        ms, _ = timed(lambda: rp.pagerank(20, 0.85, precision=prec, out=r32), reps=2)
        out[f"{name}_ms_per_iter"] = round(ms / 20, 4)
        out[f"{name}_gbs"] = round(bytes_it[name] / (ms / 20 / 1e3) / 1e9, 1)
        out[f"{name}_frac_hbm"] = round(bytes_it[name] / (ms / 20 / 1e3) / 1e9 / hbm, 4)
    if host_in is not None:
        parity["rmat25_pagerank"] = pr25_parity(n, host_in, r32, r64)
    out["rel_l1_vs_fp64_per_iter"] = [float("%.3e" % x) for x in rel]
    out["max_abs_vs_fp64_per_iter"] = [float("%.3e" % x) for x in mx]
    _, i32, h32 = rp.pagerank(1000, 0.85, precision=G.PR_FP32_KAHAN, tolerance=1e-9, l1_history=True, out=r32)
    _, i64, h64 = rp.pagerank(1000, 0.85, precision=G.PR_FP64, tolerance=1e-9, l1_history=True, out=r64)
    d = (r32 - r64).abs()
    out["to_1e-9"] = {"fp32_kahan_iters": i32, "fp64_iters": i64, "rel_l1": float("%.3e" % float(d.sum() / r64.abs().sum())),
                      "max_abs": float("%.3e" % float(d.max())), "fp32_kahan_last_l1": h32[-1] if h32 else None,
                      "fp64_last_l1": h64[-1] if h64 else None}
    rp.close()
    return out


def dropin_leg(args, srcs):
    """The reference-facing Cuda_BFS (include/GPU_csr/algorithm/GPU_BFS_csr.cuh)
    end to end on this workload, timed by the C++ driver build/dropin/
    dropin_bfs_bench as the reference's LDBC driver times it
    (LDBC_GPU_csr.cu:82-95): names in, host vector of (name, depth) out."""
    exe = os.path.join(ROOT, "build", "dropin", "dropin_bfs_bench")
    if not os.path.exists(exe):
        return {"unavailable": "build/dropin/dropin_bfs_bench not built (make dropin with REF_ROOT)"}
    cmd = [exe, str(args.scale), str(args.edge_factor), str(args.seed), ",".join(str(s) for s in srcs)]
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=600)
    except subprocess.TimeoutExpired:
        return {"unavailable": "dropin_bfs_bench exceeded 600 s"}
    line = (r.stdout.strip().splitlines() or [""])[-1]
    try:
        d = json.loads(line)
    except ValueError:
        return {"unavailable": f"dropin_bfs_bench rc={r.returncode}: {r.stderr.strip()[-300:]}"}
    d["rc"] = r.returncode
    d["note"] = ("Cuda_BFS(graph, csr, name) per source: BFS on the CSR_graph's resident copy, the depths to a "
                 "host vector (one byte each over PCIe, widened on host threads), ids -> names "
                 "(vector<pair<string,int>>); bfs_plus_copy = the same call's BFS and depth transfer without the "
                 "naming")
    return d


def rel_l1(a, b):
    return float(np.abs(a - b).sum() / np.abs(b).sum())


PR_TOL = 1e-6  # PageRank: relative L1 distance to the FP64 CPU result


def grid_parity(grid, c, dg, dgs):
    """BFS depths and SSSP distances from the centre of the 4096 x 4096 grid
    against the oracle (FIFO BFS, Dijkstra), bit for bit."""
    import oracle as O
    rp, col, w = grid.rowptr.cpu().numpy(), grid.col.cpu().numpy(), grid.w.cpu().numpy()
    og = O.Graph(grid.n, rp, col, w, False, rp, col, w)
    t0 = time.perf_counter()
    ok_bfs = bool(np.array_equal(dg.cpu().numpy(), O.bfs(og, c)))
    ok_sssp = bool(np.array_equal(dgs.cpu().numpy(), O.sssp(og, c)))
    return {"bfs_depths_equal": ok_bfs, "sssp_dist_equal": ok_sssp, "checker": "oracle (port) BFS and Dijkstra",
            "check_s": round(time.perf_counter() - t0, 1)}


def pr25_parity(n, host_in, r32, r64):
    """RMAT-25 (directed, ~10 % dangling) PageRank after 20 iterations, FP32
    ranks + Kahan rows and FP64, against the oracle's FP64 PageRank."""
    import oracle as O
    irp, icol, orp = host_in
    og = O.Graph(n, orp, np.empty(0, np.int32), None, True, irp, icol, None)
    t0 = time.perf_counter()
    ref = O.pagerank(og, 20, 0.85)
    e32, e64 = rel_l1(r32.cpu().numpy(), ref), rel_l1(r64.cpu().numpy(), ref)
    return {"iterations": 20, "fp32_kahan_rel_l1": float("%.3e" % e32), "fp64_rel_l1": float("%.3e" % e64),
            "tolerance": PR_TOL, "within_tolerance": bool(e32 <= PR_TOL and e64 <= PR_TOL),
            "checker": "oracle (port) FP64 PageRank", "check_s": round(time.perf_counter() - t0, 1)}


def tc_reference_estimate(scale=16, seed=7):
    """The reference's Tri_Counting (CPU_TC.hpp:31-60) merges row(u) with
    row(v) for every entry u -> v, so its work is sum over entries of
    deg(u) + deg(v) = 2 * sum deg^2.  It is timed on RMAT-16 (the same
    generator, seed 7) and its time per unit of sum deg^2 returned."""
    import oracle as O
    og = O.rmat_graph(scale, 16, seed, directed=False, weight_mode=0)
    d = np.diff(og.rowptr).astype(np.float64)
    r = O.Ref().load(og)
    t0 = time.perf_counter()
    r.tc()
    dt = time.perf_counter() - t0
    r.close()
    return dt / float((d * d).sum()), dt, og.m


def cpu_section(args, G, g, rg, srcs, parity, ex):
    """Parity of every algorithm on the benchmark graph, and the reference's
    CPU functions (compiled from its sources, oracle/_ref) timed on it.

    Checkers: the compiled reference itself for BFS, SSSP, WCC, PageRank and
    one CDLP iteration (the oracle port equals it bit for bit, pinned in
    tests/test_oracle_golden.py); the port (all host threads) for ten CDLP
    iterations; the oriented CPU count (oracle.tc_oriented, pinned to
    Tri_Counting in the tests) for TC, since the reference's TC is quadratic
    in the hub degrees here.  Timing follows LDBC_CPU_adj_list.cpp:113-126:
    one warm-up (a BFS over the freshly loaded graph), then one timed run of
    each function, with the reference's own threading."""
    import torch

    import oracle as O
    n, m = g.n, g.m
    nproc = os.cpu_count() or 1
    t_all = time.perf_counter()
    # GPU outputs on the benchmark graph (caller's ids).
    s0, s1 = srcs[0], srcs[1]
    gpu = {}
    gpu["bfs0"] = rg.bfs(s0)[0].cpu().numpy()
    gpu["bfs1"] = rg.bfs(s1)[0].cpu().numpy()
    gpu["sssp0"] = rg.sssp(s0)[0].cpu().numpy()
    gpu["wcc"] = rg.wcc().cpu().numpy()
    gpu["pr64"] = rg.pagerank(10, 0.85, precision=G.PR_FP64)[0].cpu().numpy()
    gpu["pr32"] = rg.pagerank(10, 0.85, precision=G.PR_FP32_KAHAN)[0].cpu().numpy()
    gpu["cdlp1"] = rg.cdlp(1).cpu().numpy()
    gpu["cdlp10"] = rg.cdlp(10).cpu().numpy()
    c64, c32, tri = rg.tc()
    gpu["tc64"], gpu["tc32"], gpu["tri"] = c64.cpu().numpy(), c32.cpu().numpy(), int(tri)
    del c64, c32
    rp, col, w = g.rowptr.cpu().numpy(), g.col.cpu().numpy(), g.w.cpu().numpy()
    og = O.Graph(n, rp, col, w, False, rp, col, w)
    deg = np.diff(rp).astype(np.int64)
    cpu = {}
    p = parity.setdefault("rmat24", {"graph": f"RMAT scale {args.scale} edge factor {args.edge_factor} "
                                             f"seed {args.seed}, undirected", "n": n, "m": m})

    def mr_of(d):
        return int(deg[d != 2**31 - 1].sum())

    if O.ref_available():
        t0 = time.perf_counter()
        r = O.Ref().load(og)
        load_s = time.perf_counter() - t0
        r.bfs(s1)  # warm-up
        kind = "reference"

        def run(fn):
            t = time.perf_counter()
            v = fn()
            return v, time.perf_counter() - t
        d, t = run(lambda: r.bfs(s0))
        p["bfs_depths_equal"] = bool(np.array_equal(d, gpu["bfs0"]))
        cpu["bfs"] = {"cpu": round(mr_of(d) / t / 1e9, 4), "gpu": ex.get("bfs_gteps_single"), "unit": "GTEPS",
                      "cores": 1, "kind": kind, "cpu_s": round(t, 2),
                      "sample": "reference CPU_BFS (CPU_BFS.hpp:10-41, single-threaded by design) from the first "
                                "benchmark source on the benchmark graph"}
        d, t = run(lambda: r.sssp(s0))
        p["sssp_dist_equal"] = bool(np.array_equal(d, gpu["sssp0"]))
        cpu["sssp"] = {"cpu": round(mr_of(d) / t / 1e9, 4), "gpu": ex.get("sssp_gteps"), "unit": "GTEPS",
                       "cores": 1, "kind": kind, "cpu_s": round(t, 2),
                       "sample": "reference CPU_shortest_paths (CPU_shortest_paths.hpp:19-64, Dijkstra, "
                                 "single-threaded) from the first benchmark source"}
        d, t = run(r.wcc)
        p["wcc_labels_equal"] = bool(np.array_equal(d, gpu["wcc"]))
        cpu["wcc"] = {"cpu": round(t * 1e3, 1), "gpu": ex.get("wcc_ms"), "unit": "ms", "cores": nproc,
                      "kind": kind, "sample": "reference CPU_connected_components (CPU_connected_components.hpp:"
                                              "12-66, hardware_concurrency threads), whole graph"}
        d, t = run(lambda: r.pagerank(10, 0.85))
        e64, e32 = rel_l1(gpu["pr64"], d), rel_l1(gpu["pr32"], d)
        p["pagerank_fp64_rel_l1"] = float("%.3e" % e64)
        p["pagerank_fp32_kahan_rel_l1"] = float("%.3e" % e32)
        p["pagerank_within_tolerance"] = bool(e64 <= PR_TOL and e32 <= PR_TOL)
        p["pagerank_tolerance"] = PR_TOL
        cpu["pagerank"] = {"cpu": round(t * 1e3 / 10, 1), "gpu": ex.get("pr_fp32_kahan_ms_per_iter"),
                           "unit": "ms per iteration", "cores": nproc, "kind": kind,
                           "sample": "reference PageRank (CPU_PageRank.hpp:12-56, 100-task pool), 10 iterations"}
        d, t = run(lambda: r.cdlp(1))
        p["cdlp_1_iteration_equal"] = bool(np.array_equal(d, gpu["cdlp1"]))
        cpu["cdlp"] = {"cpu": round(t * 1e3, 1), "gpu": ex.get("cdlp_ms_per_iter"), "unit": "ms per iteration",
                       "cores": nproc, "kind": kind,
                       "sample": "reference CDLP (CPU_Community_Detection.hpp:12-64, 100-task pool), one iteration "
                                 "(ten take ten times as long; the GPU figure is the mean of ten)"}
        r.close()
        del r
        cpu["load_s"] = round(load_s, 1)
    else:
        kind = "port"
        p["bfs_depths_equal"] = bool(np.array_equal(O.bfs(og, s0), gpu["bfs0"]))
        p["sssp_dist_equal"] = bool(np.array_equal(O.sssp(og, s0), gpu["sssp0"]))
        p["wcc_labels_equal"] = bool(np.array_equal(O.wcc(og), gpu["wcc"]))
        ref = O.pagerank(og, 10, 0.85)
        e64, e32 = rel_l1(gpu["pr64"], ref), rel_l1(gpu["pr32"], ref)
        p["pagerank_fp64_rel_l1"], p["pagerank_fp32_kahan_rel_l1"] = float("%.3e" % e64), float("%.3e" % e32)
        p["pagerank_within_tolerance"] = bool(e64 <= PR_TOL and e32 <= PR_TOL)
        p["pagerank_tolerance"] = PR_TOL
    p["bfs_second_source_equal"] = bool(np.array_equal(O.bfs(og, s1), gpu["bfs1"]))
    t0 = time.perf_counter()
    p["cdlp_10_iterations_equal"] = bool(np.array_equal(O.cdlp(og, 10), gpu["cdlp10"]))
    p["cdlp_10_check_s"] = round(time.perf_counter() - t0, 1)
    t0 = time.perf_counter()
    c, t_cpu = O.tc_oriented(og)
    p["tc_check_s"] = round(time.perf_counter() - t0, 1)
    p["tc_counts64_equal"] = bool(np.array_equal(c, gpu["tc64"]))
    p["tc_counts32_equal"] = bool(np.array_equal((c & 0xFFFFFFFF).astype(np.uint32).view(np.int32), gpu["tc32"]))
    p["tc_triangles"] = t_cpu
    p["tc_triangles_equal"] = t_cpu == gpu["tri"]
    p["checkers"] = (f"{kind} (compiled reference) for BFS, SSSP, WCC, PageRank and one CDLP iteration; oracle port "
                     "for a second BFS source and ten CDLP iterations; oriented CPU count (pinned to Tri_Counting "
                     "in the tests) for TC") if kind == "reference" else "oracle port; oriented CPU count for TC"
    if O.ref_available():
        rate, dt16, m16 = tc_reference_estimate()
        d = deg.astype(np.float64)
        est = rate * float((d * d).sum())
        cpu["tc"] = {"cpu": round(est, 0), "gpu": round(ex["tc_ms"] / 1e3, 3) if "tc_ms" in ex else None,
                     "unit": "s", "cores": 1, "kind": "reference", "estimate": True,
                     "sample": f"reference Tri_Counting (CPU_TC.hpp:31-60, single-threaded) timed on RMAT-16 "
                               f"seed 7 ({m16} entries, {dt16:.1f} s) and scaled by sum(deg^2), the merge work "
                               f"of its every-entry row intersection; the benchmark graph would take hours"}
    for k, v in cpu.items():
        if isinstance(v, dict) and v.get("gpu"):
            hi = v["unit"] == "GTEPS"
            v["gpu_over_cpu"] = round(v["gpu"] / v["cpu"], 1) if hi else round(v["cpu"] / v["gpu"], 1)
    checks = [p[k] for k in ("bfs_depths_equal", "bfs_second_source_equal", "sssp_dist_equal", "wcc_labels_equal",
                             "pagerank_within_tolerance", "cdlp_10_iterations_equal", "tc_counts64_equal",
                             "tc_counts32_equal", "tc_triangles_equal")]
    if "cdlp_1_iteration_equal" in p:
        checks.append(p["cdlp_1_iteration_equal"])
    p["all_equal"] = bool(all(checks))
    grid, pr25 = parity.get("grid4096"), parity.get("rmat25_pagerank")
    parity["all_green"] = bool(p["all_equal"] and (grid is None or (grid["bfs_depths_equal"] and grid["sssp_dist_equal"]))
                               and (pr25 is None or pr25["within_tolerance"]))
    cpu["host_threads"] = nproc
    cpu["section_s"] = round(time.perf_counter() - t_all, 1)
    return cpu


def cpu_baseline_port(g, srcs):
    """The oracle (C restatement of the reference's CPU BFS) on the host."""
    import oracle as O
    og = O.Graph(g.n, g.rowptr.cpu().numpy(), g.col.cpu().numpy(), None, False, None, None, None)
    og.in_rowptr, og.in_col = og.rowptr, og.col
    deg = np.diff(og.rowptr)
    t_tot, e_tot = 0.0, 0
    for s in srcs:
        t0 = time.perf_counter()
        d = O.bfs(og, s)
        t_tot += time.perf_counter() - t0
        e_tot += int(deg[d != 2**31 - 1].sum())
    return {"value": round(e_tot / t_tot / 1e9, 4), "unit": "GTEPS", "cores": 1, "kind": "port",
            "sample": f"BFS from {len(srcs)} of the same sources on the same graph (single-threaded FIFO BFS, "
                      f"CPU_BFS.hpp:10-41), {t_tot:.1f} s"}


# ----------------------------------------------------------- reference
def run_reference(args, world, rank):
    import oracle as O
    if rank != 0:
        return None
    if not O.ref_available():
        return {"impl": "reference", "unavailable": "oracle/_ref/libref.so was not built (reference tree absent)"}
    t0 = time.time()
    og = O.rmat_graph(args.scale, args.edge_factor, args.seed, directed=False)
    build_s = time.time() - t0
    r = O.Ref().load(og)
    srcs = pick_sources(og.rowptr, args.sources, args.seed)
    deg = np.diff(og.rowptr)
    # The reference's CPU_BFS is single-threaded; a step runs one BFS per
    # host thread at once (different sources, shared read-only graph), a
    # bounded sample of the 64-source step.
    from concurrent.futures import ThreadPoolExecutor
    threads = max(1, os.cpu_count() or 1)
    pool = ThreadPoolExecutor(max_workers=threads)

    def one(i):
        d = r.bfs(srcs[i % len(srcs)])
        return int(deg[d != 2**31 - 1].sum())
    for i in range(args.warmup):
        list(pool.map(one, range(i * threads, (i + 1) * threads)))
    t_tot, e_tot = 0.0, 0
    for i in range(args.steps):
        t = time.perf_counter()
        e_tot += sum(pool.map(one, range((args.warmup + i) * threads, (args.warmup + i + 1) * threads)))
        t_tot += time.perf_counter() - t
    pool.shutdown()
    v = e_tot / t_tot / 1e9
    return {
        "impl": "reference", "metric": METRIC, "value": round(v, 4), "unit": "GTEPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(1e3 * t_tot / args.steps, 2),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic",
        # The same workload as the GPU arm (64 sources of this graph); a
        # step here is a bounded sample of it: `threads` of the 64 sources,
        # rotating, so consecutive steps cover all of them.
        "config": {"workload": f"BFS from {len(srcs)} random non-isolated sources, undirected RMAT "
                               f"scale {args.scale} edge factor {args.edge_factor} seed {args.seed}",
                   "n": og.n, "m": og.m, "sources_per_step": len(srcs),
                   "l2": "inputs larger than L2 (col %.2f GB)" % (4 * og.m / 1e9),
                   "parallelism": f"replicas x{world}"},
        "sample_sources_per_step": threads,
        "cpu_baseline": {"value": round(v, 4), "unit": "GTEPS", "cores": threads, "kind": "reference",
                         "sample": f"reference CPU_BFS (single-threaded by design), {threads} of the 64 sources per "
                                   f"step, one per host thread at once, rotating over the 64; {args.steps} steps"},
        "e2e": {"value": round(v, 4), "unit": "GTEPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "build_s": round(build_s, 1),
    }


def run_only(args):
    """One algorithm on the seeded RMAT graph of --scale: the small cases that
    the committed ncu summaries capture (kernel names are filtered by ncu)."""
    import torch

    import graphhet_b200 as G
    g = G.rmat_graph(args.scale, args.edge_factor, args.seed)
    if args.only == "gpma":
        return gpma_only(args, G, g)
    rg = G.ResidentGraph(g)
    srcs = pick_sources(g.rowptr.cpu().numpy(), 256, args.seed)
    n = g.n
    i32 = torch.empty(n, dtype=torch.int32, device="cuda")
    f64 = torch.empty(n, dtype=torch.float64, device="cuda")
    big = None
    if args.only.startswith("msbfs"):
        big = torch.empty(256 * n, dtype=torch.int32, device="cuda")
    if args.only.startswith("mssssp"):
        big = torch.empty(256 * n, dtype=torch.float64, device="cuda")
    calls = {
        "bfs": lambda i: rg.bfs(srcs[i % len(srcs)], out=i32),
        "sssp": lambda i: rg.sssp(srcs[i % len(srcs)], out=f64),
        "wcc": lambda i: rg.wcc(out=i32),
        "pr": lambda i: rg.pagerank(10, 0.85, precision=G.PR_FP32_KAHAN, out=f64),
        "pr64": lambda i: rg.pagerank(10, 0.85, precision=G.PR_FP64, out=f64),
        "cdlp": lambda i: rg.cdlp(10, out=i32),
        "tc": lambda i: rg.tc(),
        "msbfs64": lambda i: rg.msbfs(srcs[:64], out=big),
        "msbfs256": lambda i: rg.msbfs(srcs[:256], out=big),
        "mssssp256": lambda i: rg.mssssp(srcs[:256], out=big),
    }
    fn = calls[args.only]
    for i in range(args.warmup):
        fn(i)
    torch.cuda.synchronize()
    ms, _ = timed(lambda: [fn(i) for i in range(args.steps)])
    return {"only": args.only, "scale": args.scale, "n": n, "m": g.m, "steps": args.steps,
            "ms_per_call": round(ms / max(1, args.steps), 4)}


def gpma_only(args, G, g):
    """Dynamic-graph section alone, plus the reference's CPU edits
    (graph_structure::add_edge / remove_edge, CPU_adj_list.hpp:110-128, from
    oracle/_ref) applying the same 1,000- and 100,000-update batches on this
    graph on one host thread, as the CPU baseline of the update path."""
    import torch
    sizes = tuple(int(x) for x in args.gpma_sizes.split(","))
    reps = tuple(20 if x <= 1000 else 10 if x <= 100000 else 3 for x in sizes)
    out = {"only": "gpma", "scale": args.scale, "n": g.n, "m": g.m, "gpu": gpma_section(G, g, sizes, reps)}
    sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
    import oracle as O
    if O.ref_available():
        og = O.Graph(g.n, g.rowptr.cpu().numpy(), g.col.cpu().numpy(), g.w.cpu().numpy(), False,
                     g.rowptr.cpu().numpy(), g.col.cpu().numpy(), g.w.cpu().numpy())
        r = O.Ref().load(og)
        gen = torch.Generator(device="cuda")
        gen.manual_seed(args.seed + 1)
        cpu = {}
        for size in (1000, 100000):
            k, v = gpma_batch(g, size, gen)
            k = k.cpu().numpy()
            t0 = time.perf_counter()
            r.apply_updates((k >> 32).astype(np.int32), (k & 0xFFFFFFFF).astype(np.int32), v.cpu().numpy())
            dt = time.perf_counter() - t0
            cpu[f"batch{size}_ms"] = round(dt * 1e3, 3)
            cpu[f"batch{size}_mupdates_per_s"] = round(size / dt / 1e6, 3)
        r.close()
        out["cpu_reference_graph_structure"] = dict(cpu, cores=1, kind="reference")
    return out


def main():
    args = parse()
    if args.only:
        print(json.dumps(run_only(args)), flush=True)
        return
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        out = run_reference(args, world, rank)
    else:
        out = run_ours(args, world, rank, local)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
