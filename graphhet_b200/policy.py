"""Learned schedule policy for the CSR traversals: training data, training,
evaluation.

The network (12 -> 64 -> 64 -> 20 logits in three heads: BFS direction,
top-down output format, SSSP bucket-width bin) is trained by libghb's own
kernels (``ghb_mlp_train``) and runs inside the persistent BFS kernel, where
the block that closes a level evaluates it before releasing the grid, and in
the SSSP width choice.  The reference has no counterpart: its BFS is
top-down only (GPU_BFS_csr.cuh:15-249), its BFS_pre switches direction at a
fixed n/100 frontier (GPU_BFS_pre_csr.cuh:104-118), and its SSSP has no
buckets (GPU_SSSP_csr.cuh:253-319).

Labels come from measurement.  The vertex set of BFS level L does not depend
on the directions taken before it, so one traversal can be replayed under
forced schedules (GHB_POLICY_SCHEDULE) and timed level by level inside the
persistent kernel:

  A  every level top-down, next frontier written as a queue
  B  every level top-down, next frontier written as a bitmap only (the next
     top-down level first turns it into a queue; that time is recorded apart)
  C  every level after the first bottom-up (at most PULL_LEVEL_CAP levels)

From those times a dynamic program over the frontier's form (queue or bitmap
only) gives the cheapest schedule (`oracle_schedule`); its decisions are the
labels, and the schedule itself, replayed, is the per-level oracle against
which a policy's regret is measured.  SSSP labels are the fastest of the
bucket widths 2^(k-6) x the weight rule's width, k = 0..15, timed per graph.
"""
from __future__ import annotations

import json
import math
import os
import time
from dataclasses import asdict, dataclass
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
WEIGHTS_PATH = os.path.join(_HERE, "policy_net.npz")

N_FEATURES, N_OUT, N_PARAMS = 12, 20, 6292
DELTA_BINS, DELTA_BIN_ZERO = 16, 6
# Schedule bytes: bit 0 direction, bits 1-2 top-down output (1 queue, 2 bitmap).
PUSH_QUEUE, PUSH_BITMAP, PULL = 2, 4, 1
PULL_LEVEL_CAP = 96
# Trace columns (include/ghb.h).
T_DIR, T_MS, T_FMT, T_COMP, T_NET = 12, 13, 20, 21, 22


# ------------------------------------------------------------ graph family
@dataclass
class GraphSpec:
    kind: str          # rmat | er | grid | powerlaw
    scale: int         # log2 of the vertex count
    param: float       # rmat: a; er: mean degree; grid: aspect log2; powerlaw: exponent
    edge_factor: int   # generated edges per vertex (rmat, powerlaw)
    seed: int


def training_specs(count: int = 400, seed: int = 4) -> List[GraphSpec]:
    """The training family: RMAT with a in [.45, .65], Erdos-Renyi, grids and
    Chung-Lu power-law graphs with exponent in [2.1, 2.8], scales 16-22,
    cycled in that order.  Held out: the scale-24 RMAT and the 4096x4096 grid."""
    rng = np.random.default_rng(seed)
    kinds = ["rmat", "er", "grid", "powerlaw"]
    out = []
    for i in range(count):
        kind = kinds[i % 4]
        scale = int(rng.integers(16, 23))
        if kind == "rmat":
            param, ef = float(rng.uniform(0.45, 0.65)), int(rng.choice([4, 8, 16, 32]))
        elif kind == "er":
            param, ef = float(rng.uniform(2.0, 32.0)), 0
        elif kind == "grid":
            param, ef = float(rng.integers(0, 3)), 0
        else:
            param, ef = float(rng.uniform(2.1, 2.8)), int(rng.choice([2, 4, 8, 16]))
        out.append(GraphSpec(kind, scale, param, ef, int(rng.integers(1, 2**31))))
    return out


def build_graph(spec: GraphSpec, weighted: bool = True):
    """CSRGraph of a spec on the current CUDA device (undirected, weights
    U(0,1] except grids, which get integers in [1, 100])."""
    import graphhet_b200 as G
    wm = G.WEIGHT_UNIFORM01 if weighted else G.WEIGHT_NONE
    n = 1 << spec.scale
    if spec.kind == "rmat":
        a = spec.param
        b = c = (1.0 - a - 0.05) / 2.0
        return G.rmat_graph(spec.scale, spec.edge_factor, spec.seed, a=a, b=b, c=c, weight_mode=wm)
    if spec.kind == "er":
        src, dst = G.gen_er(n, int(n * spec.param / 2), spec.seed)
        return G.make_graph(n, src, dst, False, weight_mode=wm, weight_seed=spec.seed)
    if spec.kind == "grid":
        r = spec.scale // 2 - int(spec.param)
        return G.grid_graph(1 << r, 1 << (spec.scale - r), weight_seed=spec.seed)
    src, dst = G.gen_powerlaw(spec.scale, n * spec.edge_factor, spec.param, spec.seed)
    return G.make_graph(n, src, dst, False, weight_mode=wm, weight_seed=spec.seed)


def pick_sources(g, k: int, seed: int) -> List[int]:
    """k distinct vertices with at least one entry, seeded."""
    import torch
    deg = (g.rowptr[1:] - g.rowptr[:-1]).cpu().numpy()
    cand = np.nonzero(deg > 0)[0]
    if cand.size == 0:
        return []
    rng = np.random.default_rng(seed)
    return [int(x) for x in rng.choice(cand, size=min(k, cand.size), replace=False)]


# ------------------------------------------------------ per-level oracle
def oracle_schedule(t_queue: Sequence[float], t_bitmap: Sequence[float], t_comp: Sequence[float],
                    t_pull: Sequence[float]) -> Tuple[List[int], List[float], float]:
    """Cheapest schedule for one traversal from per-level costs.

    t_queue[L]   top-down level L writing the next frontier as a queue
    t_bitmap[L]  top-down level L writing it as a bitmap only (expansion)
    t_comp[L]    turning frontier L from a bitmap into a queue
    t_pull[L]    bottom-up level L (inf where not timed)
    Level 0's frontier is a queue.  A top-down level needs a queue (paying
    t_comp if the frontier is a bitmap); a bottom-up level reads the bitmap,
    which always exists, and leaves a bitmap.  Returns the schedule bytes, the
    chosen cost of each level (compaction included) and the total."""
    L = len(t_queue)
    INF = float("inf")
    # V[l][s]: cheapest cost of levels l.. with frontier l in form s (0 queue, 1 bitmap).
    V = [[0.0, 0.0] for _ in range(L + 1)]
    act = [[None, None] for _ in range(L)]
    for l in range(L - 1, -1, -1):
        for s in (0, 1):
            comp = 0.0 if s == 0 else (t_comp[l] if t_comp[l] >= 0 else 0.0)
            opts = [(comp + t_queue[l] + V[l + 1][0], PUSH_QUEUE),
                    (comp + t_bitmap[l] + V[l + 1][1], PUSH_BITMAP),
                    ((t_pull[l] if l > 0 else INF) + V[l + 1][1], PULL)]
            best = min(opts, key=lambda x: x[0])
            V[l][s], act[l][s] = best
    sched, cost, s = [], [], 0
    for l in range(L):
        a = act[l][s]
        comp = 0.0 if s == 0 else (t_comp[l] if t_comp[l] >= 0 else 0.0)
        c = {PUSH_QUEUE: comp + t_queue[l], PUSH_BITMAP: comp + t_bitmap[l], PULL: t_pull[l]}[a]
        sched.append(a)
        cost.append(c)
        s = 0 if a == PUSH_QUEUE else 1
    return sched, cost, V[0][0]


def level_weights(r: dict, sched: Sequence[int], total: float) -> np.ndarray:
    """Importance of each level's decision: what a wrong direction or format
    costs at that level (from the replayed times), as a share of the whole
    traversal's oracle time, times the number of levels (mean 1 when every
    level matters equally)."""
    L = len(sched)
    w = np.zeros(L)
    for l in range(L):
        push = min(r["t_queue"][l], r["t_bitmap"][l] + (r["t_comp"][l + 1] if l + 1 < L else 0.0))
        pull = r["t_pull"][l]
        gap_dir = abs(pull - push) if np.isfinite(pull) else 0.0
        gap_fmt = abs(r["t_queue"][l] - (r["t_bitmap"][l] + (r["t_comp"][l + 1] if l + 1 < L else 0.0)))
        w[l] = (gap_dir + gap_fmt) / max(total, 1e-9) * L
    return w


def level_rows(trace_a: np.ndarray, sched: Sequence[int], cost: Sequence[float],
               max_rows: int = 48, weights: Optional[np.ndarray] = None):
    """Training rows of one traversal: the features of frontier L (the same in
    every replay) with the history feature (9, previous direction) taken from
    the oracle schedule, and the labels
    (direction, top-down output format).  Level 0 is skipped: the kernel
    decides it without the network.  A long traversal (a grid's thousands of
    levels) gives its first max_rows/2 levels and evenly spaced others, so
    that it does not outweigh the rest of the family."""
    X, Y = [], []
    levels = list(range(1, len(sched)))
    if len(levels) > max_rows:
        head = levels[: max_rows // 2]
        rest = levels[max_rows // 2:]
        pick = np.linspace(0, len(rest) - 1, max_rows - len(head)).round().astype(int)
        levels = head + [rest[i] for i in sorted(set(pick.tolist()))]
    W = []
    for l in levels:
        W.append(1.0 if weights is None else float(weights[l]))
        f = trace_a[l, :N_FEATURES].astype(np.float32).copy()
        f[9] = 1.0 if sched[l - 1] == PULL else 0.0
        d = 1 if sched[l] == PULL else 0
        fm = -1 if d else (0 if sched[l] == PUSH_QUEUE else 1)
        X.append(f)
        Y.append([d, fm, -1])
    if not X:
        if weights is None:
            return np.zeros((0, N_FEATURES), np.float32), np.zeros((0, 3), np.int32)
        return np.zeros((0, N_FEATURES), np.float32), np.zeros((0, 3), np.int32), np.zeros(0, np.float32)
    if weights is None:
        return np.asarray(X, np.float32), np.asarray(Y, np.int32)
    return np.asarray(X, np.float32), np.asarray(Y, np.int32), np.asarray(W, np.float32)


def replay_costs(rg, src: int):
    """Run schedules A, B, C on one source; per-level cost table and run A's
    trace (features).  Returns None when the traversal has one level."""
    import graphhet_b200 as G
    cap = 1 << 15
    _, st_a, ta = rg.bfs(src, policy=G.POLICY_SCHEDULE, schedule=[PUSH_QUEUE] * cap, trace_cap=cap)
    levels = ta.shape[0]
    if levels < 2:
        return None
    _, _, tb = rg.bfs(src, policy=G.POLICY_SCHEDULE, schedule=[PUSH_BITMAP] * levels, trace_cap=levels)
    npull = min(levels, PULL_LEVEL_CAP)
    sched_c = [PUSH_QUEUE] + [PULL] * (npull - 1) + [PUSH_QUEUE] * (levels - npull)
    _, _, tc = rg.bfs(src, policy=G.POLICY_SCHEDULE, schedule=sched_c, trace_cap=levels)
    t_q = ta[:, T_MS].astype(np.float64)
    comp_b = np.where(tb[:, T_COMP] >= 0, tb[:, T_COMP], 0.0).astype(np.float64)
    t_b = tb[:, T_MS].astype(np.float64) - comp_b
    # Frontier l of run B is a bitmap for l >= 1, so run B timed every compaction.
    t_comp = comp_b.copy()
    t_p = np.full(levels, np.inf)
    t_p[1:npull] = tc[1:npull, T_MS]
    return dict(t_queue=t_q, t_bitmap=t_b, t_comp=t_comp, t_pull=t_p, trace=ta, levels=levels,
                m_r=st_a["edges_reached"])


# ------------------------------------------------------------ SSSP labels
def sssp_rows(rg, srcs: Sequence[int], max_buckets: float = 4096.0, max_ms: float = 2000.0):
    """Rows for the width head from several sources of one graph: each
    source's features, all labelled with the width bin that is fastest over
    all of them (the sum of their times: one timing per source and bin is
    noisy, the graph's best width is not), weighted by the rule's width's
    excess time over that bin.  Bins whose width would give more than
    max_buckets buckets over a source's largest finite distance are not run
    and cannot win.  Returns (features[k, 12], label, weight, times[k, 16])
    or None."""
    import torch
    feats, T = [], []
    for src in srcs:
        d0, st0, row = rg.sssp(src, trace=True)
        base = float(row[14])
        fin = d0[d0 < 1e300]
        dmax = float(fin.max().item()) if fin.numel() else 0.0
        times = np.full(DELTA_BINS, np.inf)
        for k in range(DELTA_BINS):
            delta = base * 2.0 ** (k - DELTA_BIN_ZERO)
            if dmax / delta > max_buckets:
                continue
            d, st = rg.sssp(src, delta=delta)
            times[k] = st["device_ms"]
            if not torch.equal(d, d0):
                raise RuntimeError("SSSP distances changed with the bucket width")
            if st["device_ms"] > max_ms:
                break
        feats.append(row[:N_FEATURES].astype(np.float32))
        T.append(times)
    if not feats:
        return None
    T = np.array(T)
    tot = T.sum(0)
    if not np.isfinite(tot).any():
        return None
    lab = int(np.argmin(tot))
    rule = tot[DELTA_BIN_ZERO] if np.isfinite(tot[DELTA_BIN_ZERO]) else np.nanmax(np.where(np.isfinite(tot), tot, np.nan))
    weight = float(np.clip(rule / tot[lab] - 1.0, 0.05, 10.0))
    return np.stack(feats), lab, weight, T


# ------------------------------------------------------------- collection
def collect(specs: Sequence[GraphSpec], bfs_sources: int = 6, grid_sources: int = 2, sssp_every: int = 1,
            sssp_max_scale: int = 22, sssp_sources: int = 3,
            log=print) -> Dict[str, np.ndarray]:
    """Training rows from every graph of `specs` (needs a GPU)."""
    import torch
    import graphhet_b200 as G
    Xs, Ys, Ws, meta = [], [], [], []
    t0 = time.time()
    for gi, spec in enumerate(specs):
        g = build_graph(spec)
        rg = G.ResidentGraph(g)
        # Grids give many near-identical levels per source: fewer sources.
        srcs = pick_sources(g, grid_sources if spec.kind == "grid" else bfs_sources, spec.seed)
        nrows = 0
        for s in srcs:
            rg.bfs(s)  # warm-up (scratch, first-touch)
            r = replay_costs(rg, s)
            if r is None:
                continue
            sched, cost, total = oracle_schedule(r["t_queue"], r["t_bitmap"], r["t_comp"], r["t_pull"])
            X, Y, W = level_rows(r["trace"], sched, cost, weights=level_weights(r, sched, total))
            Xs.append(X)
            Ys.append(Y)
            Ws.append(W)
            nrows += len(X)
        if gi % sssp_every == 0 and spec.scale <= sssp_max_scale and srcs:
            out = sssp_rows(rg, srcs[:sssp_sources])
            if out is not None:
                f, lab, wt, _ = out
                Xs.append(f)
                Ys.append(np.tile(np.array([[-1, -1, lab]], np.int32), (len(f), 1)))
                Ws.append(np.full(len(f), wt, np.float32))
                nrows += len(f)
        meta.append(dict(asdict(spec), rows=nrows, n=g.n, m=int(g.m)))
        rg.close()
        del rg, g
        torch.cuda.empty_cache()
        if log and (gi % 20 == 0 or gi == len(specs) - 1):
            log("graph %d/%d %s scale %d rows %d (%.0f s)" % (gi + 1, len(specs), spec.kind, spec.scale, nrows,
                                                              time.time() - t0))
    W = np.concatenate(Ws).astype(np.float32)
    bfs = np.concatenate(Ys)[:, 0] >= 0
    # Normalise the BFS rows' weights to mean 1 and bound them.
    if bfs.any():
        W[bfs] = np.clip(W[bfs] / max(W[bfs].mean(), 1e-12), 0.02, 50.0)
    return dict(X=np.concatenate(Xs).astype(np.float32), Y=np.concatenate(Ys).astype(np.int32), W=W,
                meta=np.array(json.dumps(meta)))


# --------------------------------------------------------------- training
def init_params(seed: int = 0) -> np.ndarray:
    """He-initialised weights, zero biases, in the kernels' layout."""
    rng = np.random.default_rng(seed)
    parts = []
    for fan_in, fan_out in [(12, 64), (64, 64), (64, 20)]:
        parts.append(rng.normal(0.0, math.sqrt(2.0 / fan_in), size=fan_in * fan_out))
        parts.append(np.zeros(fan_out))
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == N_PARAMS
    return p


def norm_of(X: np.ndarray) -> np.ndarray:
    mu = X.mean(0)
    sd = X.std(0)
    return np.concatenate([mu, 1.0 / np.maximum(sd, 1e-3)]).astype(np.float32)


def train(X: np.ndarray, Y: np.ndarray, epochs: int = 3000, lr: float = 3e-3, seed: int = 0,
          W: Optional[np.ndarray] = None):
    """Full-batch Adam on the GPU with libghb's MLP kernels, rows weighted by
    W (what a wrong decision there costs).  Returns (params, norm, loss
    history)."""
    import torch
    import graphhet_b200 as G
    norm = norm_of(X)
    p = torch.from_numpy(init_params(seed)).cuda()
    w = torch.from_numpy(W.astype(np.float32)).cuda() if W is not None else None
    hist = G.mlp_train(p, torch.from_numpy(norm).cuda(), torch.from_numpy(X).cuda(), torch.from_numpy(Y).cuda(),
                       epochs=epochs, lr=lr, weight=w)
    return p.cpu().numpy(), norm, np.asarray(hist, np.float32)


def predict(params: np.ndarray, norm: np.ndarray, X: np.ndarray) -> np.ndarray:
    """Logits through ghb_mlp_forward (GPU)."""
    import torch
    import graphhet_b200 as G
    return G.mlp_forward(torch.from_numpy(params).cuda(), torch.from_numpy(norm).cuda(),
                         torch.from_numpy(X.astype(np.float32)).cuda()).cpu().numpy()


def accuracy(params, norm, X, Y) -> Dict[str, float]:
    z = predict(params, norm, X)
    out = {}
    for h, (a, b), name in [(0, (0, 2), "dir"), (1, (2, 4), "fmt"), (2, (4, 20), "delta")]:
        keep = Y[:, h] >= 0
        if keep.any():
            out[name] = float((z[keep, a:b].argmax(1) == Y[keep, h]).mean())
    return out


def save(path: str, params, norm, info: dict) -> None:
    np.savez(path, params=params.astype(np.float32), norm=norm.astype(np.float32), info=np.array(json.dumps(info)))


def load(path: str = WEIGHTS_PATH):
    z = np.load(path)
    return z["params"], z["norm"], json.loads(str(z["info"]))


def install(path: str = WEIGHTS_PATH) -> dict:
    """Install the trained network for POLICY_LEARNED (this process), and
    the multi-source pass's direction model when it has been trained."""
    import graphhet_b200 as G
    params, norm, info = load(path)
    G.policy_load(params, norm)
    if os.path.exists(MS_WEIGHTS_PATH):
        ms_install()
    return info


# ------------------------------------------- multi-source direction model
MS_WEIGHTS_PATH = os.path.join(_HERE, "policy_ms.npz")
MS_FEATURES = 8


def ms_features(mf, active, prev_active, visits, n, m, k, level, prev_pull) -> np.ndarray:
    """The multi-source pass's level features, as the kernel computes them
    (ms_level_features in csrc/msbfs.cu)."""
    tiny = 1.0 / 1073741824.0
    return np.array([math.log2(mf / m + tiny), math.log2(active / n + tiny), math.log2(m / n + tiny),
                     math.log2(k), min(level, 32) * 0.125, math.log2(visits / n + tiny), float(prev_pull),
                     math.log2((active + 1.0) / (prev_active + 1.0))], dtype=np.float64)


def ms_rows(t_push: np.ndarray, t_pull: np.ndarray, trace: np.ndarray, n: int, m: int, k: int,
            prev_dirs: Sequence[int]) -> Tuple[np.ndarray, np.ndarray, np.ndarray]:
    """Training rows of one pass: row r decides level r + 1 from the frontier
    it expands (trace row r, columns 2-3), the frontier before it and the
    frontiers visited so far.  Label: 1 where the level pulled faster;
    weight: what the wrong direction costs there (ms).  prev_dirs[r] is the
    direction the level before took in the run whose trace is given."""
    X, y, w = [], [], []
    visits = 0.0
    prev = 0.0
    for r in range(len(trace)):
        active, mf = float(trace[r, 2]), float(trace[r, 3])
        visits += active
        X.append(ms_features(mf, active, prev, visits, n, m, k, r + 1, prev_dirs[r]))
        y.append(1.0 if t_pull[r] < t_push[r] else 0.0)
        w.append(abs(float(t_pull[r]) - float(t_push[r])))
        prev = active
    return np.array(X), np.array(y), np.array(w)


def fit_ms(X: np.ndarray, y: np.ndarray, w: np.ndarray, epochs: int = 20000, lr: float = 0.05,
           l2: float = 1e-3) -> np.ndarray:
    """Weighted logistic regression (bias + one weight per feature) by
    gradient descent on the host; returns the 9 kernel weights."""
    Xb = np.hstack([np.ones((len(X), 1)), X])
    ww = w / max(w.mean(), 1e-12)
    theta = np.zeros(Xb.shape[1])
    for _ in range(epochs):
        p = 1.0 / (1.0 + np.exp(-np.clip(Xb @ theta, -40, 40)))
        g = Xb.T @ ((p - y) * ww) / len(y) + l2 * np.r_[0.0, theta[1:]]
        theta -= lr * g
    return theta.astype(np.float32)


def ms_install(path: str = MS_WEIGHTS_PATH) -> np.ndarray:
    """Load the multi-source direction model into the library (this process);
    a workspace uses it where "ms_learned" is 1."""
    import ctypes
    import graphhet_b200 as G
    wts = np.ascontiguousarray(np.load(path)["weights"].astype(np.float32))
    G._check(G.lib().ghb_ms_policy_load(wts.ctypes.data_as(ctypes.c_void_p), len(wts)), "ghb_ms_policy_load")
    return wts


# ------------------------------------------------------------- evaluation
def regret(rg, sources: Sequence[int], repeats: int = 3) -> Dict[str, float]:
    """Measured regret of the heuristic and the learned policy against the
    per-level oracle schedule on `rg` (needs an installed network): each
    policy's persistent BFS time over the sources (median of `repeats`) ÷ the
    oracle schedule's time, minus one.  Also the oracle's own estimate from
    the cost table."""
    import graphhet_b200 as G

    def timed(src, **kw):
        ts = []
        for _ in range(repeats):
            _, st = rg.bfs(src, **kw)
            ts.append(st["device_ms"])
        return float(np.median(ts)), st

    tot = dict(heuristic=0.0, learned=0.0, oracle=0.0, beamer14=0.0, table=0.0)
    for s in sources:
        rg.bfs(s)
        r = replay_costs(rg, s)
        if r is None:
            continue
        sched, cost, total = oracle_schedule(r["t_queue"], r["t_bitmap"], r["t_comp"], r["t_pull"])
        tot["table"] += total
        tot["oracle"] += timed(s, policy=G.POLICY_SCHEDULE, schedule=sched)[0]
        tot["heuristic"] += timed(s, policy=G.POLICY_HEURISTIC)[0]
        # The classic rule: alpha 14, beta 24, no frontier guard.
        tot["beamer14"] += timed(s, policy=G.POLICY_HEURISTIC, alpha=14.0, beta=24.0, gamma=1e30)[0]
        tot["learned"] += timed(s, policy=G.POLICY_LEARNED)[0]
    o = tot["oracle"]
    return dict(ms=tot, regret_heuristic=tot["heuristic"] / o - 1.0, regret_learned=tot["learned"] / o - 1.0,
                regret_beamer14=tot["beamer14"] / o - 1.0)


def ms_regret(rg, sources: Sequence[int], repeats: int = 3, learned: bool = False) -> Dict[str, object]:
    """Regret of the multi-source pass's direction rule against the
    per-level oracle: a level finds the same vertices pushed or pulled, so
    the pass is timed level by level under all-push and all-pull schedules
    (the smallest of `repeats` times per level) and the oracle takes each
    level's cheaper direction.  Returns the level times, the rule's and the
    oracle's totals (ms), the oracle schedule run as a check, and the
    rule's regret; with `learned`, also the installed direction model's
    (workspace knob ms_learned on the default workspace)."""
    _, st, _ = rg.msbfs_ex(sources, trace_cap=1)
    levels = int(st["levels"])
    cap = max(levels, 1)

    def run(schedule):
        best, dirs = None, None
        for _ in range(repeats):
            _, _, tr = rg.msbfs_ex(sources, schedule=schedule, trace_cap=cap)
            t = tr[:, 1].astype(np.float64)
            best = t if best is None else np.minimum(best, t)
            dirs = tr[:, 0].astype(np.int32)
        return best, dirs

    import graphhet_b200 as G
    t_rule, d_rule = run(None)
    t_push, _ = run([0] * (levels + 1))
    t_pull, _ = run([1] * (levels + 1))
    best = np.where(t_pull < t_push, 1, 0).astype(np.int32)
    oracle = float(np.minimum(t_push, t_pull).sum())
    # Level L (trace row L - 1) takes schedule[L - 1].
    t_sched, _ = run(best.tolist())
    rule = float(t_rule.sum())
    out = dict(levels=levels, rule_dirs=d_rule.tolist(), oracle_dirs=best.tolist(),
               ms=dict(rule=rule, oracle=oracle, oracle_run=float(t_sched.sum()), push=float(t_push.sum()),
                       pull=float(t_pull.sum())),
               regret_rule=rule / oracle - 1.0)
    if learned:
        G.tune_set("ms_learned", 1)
        try:
            t_l, d_l = run(None)
        finally:
            G.tune_set("ms_learned", 0)
        out["learned_dirs"] = d_l.tolist()
        out["ms"]["learned"] = float(t_l.sum())
        out["regret_learned"] = float(t_l.sum()) / oracle - 1.0
    return out


def collect_ms(specs: Sequence[GraphSpec], ks: Sequence[int] = (16, 64, 256), max_scale: int = 21,
               repeats: int = 2, log=print) -> Dict[str, np.ndarray]:
    """Rows for the multi-source direction model: every graph of `specs` up
    to max_scale, one pass of k seeded sources per k, timed level by level
    under all-push and all-pull schedules (the smallest of `repeats` runs)."""
    import torch
    import graphhet_b200 as G
    Xs, ys, ws_, gs, rs = [], [], [], [], []
    run = 0
    t0 = time.time()
    for gi, spec in enumerate(specs):
        if spec.scale > max_scale:
            continue
        g = build_graph(spec, weighted=False)
        rg = G.ResidentGraph(g)
        for k in ks:
            srcs = pick_sources(g, k, spec.seed + k)
            if len(srcs) < 2:
                continue
            _, st, _ = rg.msbfs_ex(srcs, trace_cap=1)
            levels = int(st["levels"])
            if levels < 1:
                continue
            times, traces = {}, {}
            for d in (0, 1):
                best = None
                for _ in range(repeats):
                    _, _, tr = rg.msbfs_ex(srcs, schedule=[d] * (levels + 1), trace_cap=levels)
                    t = tr[:, 1].astype(np.float64)
                    best = t if best is None else np.minimum(best, t)
                times[d], traces[d] = best, tr
            # The previous direction is a feature: rows from both runs.
            for d in (0, 1):
                X, y, w = ms_rows(times[0], times[1], traces[d], g.n, g.m, len(srcs), [d] * levels)
                if d == 1:
                    X[0, 6] = 0.0  # level 1 follows the set-up, not a pull
                Xs.append(X)
                ys.append(y)
                ws_.append(w)
                gs.append(np.full(len(y), gi, np.int32))
                rs.append(np.full(len(y), run, np.int32))
            run += 1
        rg.close()
        del rg, g
        torch.cuda.empty_cache()
        if log and gi % 10 == 0:
            log("ms graph %d/%d %s scale %d (%.0f s)" % (gi + 1, len(specs), spec.kind, spec.scale, time.time() - t0))
    return dict(X=np.concatenate(Xs), y=np.concatenate(ys), w=np.concatenate(ws_), G=np.concatenate(gs),
                R=np.concatenate(rs))


def collect_sssp(specs: Sequence[GraphSpec], sssp_max_scale: int = 22, sssp_sources: int = 3,
                 log=print) -> Dict[str, np.ndarray]:
    """Width-head rows only (sssp_rows on every graph of `specs` up to
    sssp_max_scale), timed with the current SSSP kernels; G[i] is the index
    of the graph that row i came from."""
    import torch
    import graphhet_b200 as G
    Xs, Ls, Ws, Gs = [], [], [], []
    t0 = time.time()
    for gi, spec in enumerate(specs):
        if spec.scale > sssp_max_scale:
            continue
        g = build_graph(spec)
        rg = G.ResidentGraph(g)
        srcs = pick_sources(g, sssp_sources, spec.seed)
        out = sssp_rows(rg, srcs) if srcs else None
        if out is not None:
            f, lab, wt, _ = out
            Xs.append(f)
            Ls.append(np.full(len(f), lab, np.int32))
            Ws.append(np.full(len(f), wt, np.float32))
            Gs.append(np.full(len(f), gi, np.int32))
        rg.close()
        del rg, g
        torch.cuda.empty_cache()
        if log and (gi % 20 == 0 or gi == len(specs) - 1):
            log("graph %d/%d %s scale %d (%.0f s)" % (gi + 1, len(specs), spec.kind, spec.scale, time.time() - t0))
    return dict(X=np.concatenate(Xs).astype(np.float32), L=np.concatenate(Ls), W=np.concatenate(Ws),
                G=np.concatenate(Gs))


def hidden(params: np.ndarray, norm: np.ndarray, X: np.ndarray) -> np.ndarray:
    """The network's second hidden layer (ReLU) for rows X, on the host."""
    p = params.astype(np.float64)
    o = 0
    W1 = p[o:o + 12 * 64].reshape(12, 64); o += 12 * 64
    b1 = p[o:o + 64]; o += 64
    W2 = p[o:o + 64 * 64].reshape(64, 64); o += 64 * 64
    b2 = p[o:o + 64]
    x = (X.astype(np.float64) - norm[:12]) * norm[12:]
    h1 = np.maximum(x @ W1 + b1, 0.0)
    return np.maximum(h1 @ W2 + b2, 0.0)


def refit_width_head(params: np.ndarray, norm: np.ndarray, X: np.ndarray, L: np.ndarray, W: np.ndarray,
                     epochs: int = 4000, lr: float = 1e-2, l2: float = 1e-4) -> np.ndarray:
    """New weights for the width head only: weighted softmax regression of
    the labels L (bins 0..15) on the fixed hidden layer, by Adam on the host.
    The BFS heads and the shared layers keep their values, so every BFS
    decision of the network is unchanged."""
    H = hidden(params, norm, X)
    n, k = H.shape[0], DELTA_BINS
    o3 = 12 * 64 + 64 + 64 * 64 + 64
    W3 = params[o3:o3 + 64 * 20].astype(np.float64).reshape(64, 20)
    b3 = params[o3 + 64 * 20:o3 + 64 * 20 + 20].astype(np.float64)
    A, c = W3[:, 4:20].copy(), b3[4:20].copy()
    Y = np.zeros((n, k))
    Y[np.arange(n), L] = 1.0
    w = (W / W.mean()).reshape(-1, 1)
    mA, vA, mc, vc = np.zeros_like(A), np.zeros_like(A), np.zeros_like(c), np.zeros_like(c)
    for t in range(1, epochs + 1):
        z = H @ A + c
        z -= z.max(1, keepdims=True)
        pz = np.exp(z)
        pz /= pz.sum(1, keepdims=True)
        g = (pz - Y) * w / n
        gA = H.T @ g + l2 * A
        gc = g.sum(0)
        for prm, grd, m1, m2 in ((A, gA, mA, vA), (c, gc, mc, vc)):
            m1 *= 0.9
            m1 += 0.1 * grd
            m2 *= 0.999
            m2 += 0.001 * grd * grd
            prm -= lr * (m1 / (1 - 0.9 ** t)) / (np.sqrt(m2 / (1 - 0.999 ** t)) + 1e-8)
    out = params.astype(np.float32).copy()
    W3[:, 4:20] = A
    b3[4:20] = c
    out[o3:o3 + 64 * 20] = W3.reshape(-1).astype(np.float32)
    out[o3 + 64 * 20:o3 + 64 * 20 + 20] = b3.astype(np.float32)
    return out


def width_accuracy(params, norm, X, L) -> float:
    H = hidden(params, norm, X)
    o3 = 12 * 64 + 64 + 64 * 64 + 64
    W3 = params[o3:o3 + 64 * 20].astype(np.float64).reshape(64, 20)
    b3 = params[o3 + 64 * 20:o3 + 64 * 20 + 20].astype(np.float64)
    return float(((H @ W3[:, 4:20] + b3[4:20]).argmax(1) == L).mean())


def main(argv=None) -> int:
    import argparse
    import torch
    ap = argparse.ArgumentParser(description="collect traces, train the schedule policy, save it")
    ap.add_argument("--graphs", type=int, default=400)
    ap.add_argument("--epochs", type=int, default=3000)
    ap.add_argument("--lr", type=float, default=3e-3)
    ap.add_argument("--out", default=WEIGHTS_PATH)
    ap.add_argument("--data", default=None, help="save / reuse the collected rows (.npz)")
    ap.add_argument("--refit-width", action="store_true",
                    help="re-time the SSSP widths on the training graphs with the current kernels and refit the "
                         "width head of the installed network (the BFS heads are kept)")
    ap.add_argument("--ms-steer", action="store_true",
                    help="time the multi-source pass's levels under all-push and all-pull schedules on the "
                         "training graphs (scale <= 20) and fit its direction model (policy_ms.npz)")
    a = ap.parse_args(argv)
    if a.ms_steer:
        if a.data and os.path.exists(a.data):
            z = np.load(a.data)
            d = dict(X=z["X"], y=z["y"], w=z["w"], G=z["G"], R=z["R"] if "R" in z else z["G"])
        else:
            d = collect_ms(training_specs(a.graphs))
            if a.data:
                np.savez(a.data, **d)
        # Every pass (graph, source count) weighs the same in total, so the
        # grids' thousands of levels do not outvote the few levels of the
        # low-diameter graphs; inside a pass a level weighs what its wrong
        # direction costs.
        run_sum = np.bincount(d["R"], weights=d["w"])
        d["w"] = d["w"] / np.maximum(run_sum[d["R"]], 1e-12)
        val = d["G"] % 10 == 0  # every tenth graph held out

        def wacc(th, X, y, w):  # accuracy weighted by what a wrong choice costs
            pred = (np.hstack([np.ones((len(X), 1)), X]) @ th) > 0
            return float((w * (pred == (y > 0.5))).sum() / max(w.sum(), 1e-12))

        th = fit_ms(d["X"][~val], d["y"][~val], d["w"][~val])
        acc = dict(train=wacc(th, d["X"][~val], d["y"][~val], d["w"][~val]),
                   val=wacc(th, d["X"][val], d["y"][val], d["w"][val]),
                   always_pull_val=float((d["w"][val] * (d["y"][val] > 0.5)).sum() / max(d["w"][val].sum(), 1e-12)))
        th_all = fit_ms(d["X"], d["y"], d["w"])
        info = dict(rows=int(len(d["y"])), graphs=int(len(np.unique(d["G"]))), pull_share=float(d["y"].mean()),
                    weighted_accuracy=acc)
        np.savez(MS_WEIGHTS_PATH, weights=th_all, info=json.dumps(info))
        print(json.dumps(dict(info, weights=th_all.tolist())))
        return 0
    if a.refit_width:
        params, norm, info = load(WEIGHTS_PATH)
        if a.data and os.path.exists(a.data):
            z = np.load(a.data)
            d = dict(X=z["X"], L=z["L"], W=z["W"], G=z["G"])
        else:
            d = collect_sssp(training_specs(a.graphs))
            if a.data:
                np.savez(a.data, **d)
        val = d["G"] % 10 == 0  # every tenth graph held out
        p_tr = refit_width_head(params, norm, d["X"][~val], d["L"][~val], d["W"][~val])
        acc = dict(before_train=width_accuracy(params, norm, d["X"][~val], d["L"][~val]),
                   before_val=width_accuracy(params, norm, d["X"][val], d["L"][val]),
                   after_train=width_accuracy(p_tr, norm, d["X"][~val], d["L"][~val]),
                   after_val=width_accuracy(p_tr, norm, d["X"][val], d["L"][val]))
        p_all = refit_width_head(params, norm, d["X"], d["L"], d["W"])
        info = dict(info, width_refit=dict(rows=int(len(d["X"])), graphs=int(len(np.unique(d["G"]))),
                                           accuracy=acc, label_hist=np.bincount(d["L"], minlength=DELTA_BINS).tolist(),
                                           kernel="one-launch SSSP"))
        save(a.out, p_all, norm, info)
        print(json.dumps(info["width_refit"]))
        return 0
    if a.data and os.path.exists(a.data):
        z = np.load(a.data)
        data = dict(X=z["X"], Y=z["Y"], W=z["W"] if "W" in z else None, meta=z["meta"])
    else:
        data = collect(training_specs(a.graphs))
        if a.data:
            np.savez(a.data, **data)
    X, Y, W = data["X"], data["Y"], data.get("W")
    # Hold out every tenth row for validation accuracy.
    idx = np.arange(len(X))
    val = idx % 10 == 0
    params, norm, hist = train(X[~val], Y[~val], epochs=a.epochs, lr=a.lr, W=W[~val] if W is not None else None)
    acc_tr, acc_val = accuracy(params, norm, X[~val], Y[~val]), accuracy(params, norm, X[val], Y[val])
    params, norm, hist_all = train(X, Y, epochs=a.epochs, lr=a.lr, W=W)
    info = dict(graphs=a.graphs, rows=int(len(X)), bfs_rows=int((Y[:, 0] >= 0).sum()),
                sssp_rows=int((Y[:, 2] >= 0).sum()), pull_frac=float((Y[:, 0] == 1).sum() / max(1, (Y[:, 0] >= 0).sum())),
                epochs=a.epochs, lr=a.lr, loss_first=float(hist_all[0]), loss_last=float(hist_all[-1]),
                acc_train=acc_tr, acc_val=acc_val)
    save(a.out, params, norm, info)
    print(json.dumps(info))
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
