"""TEST INFRASTRUCTURE ONLY: CPU checkers for the GPU path.

* ``port``: the C restatement in oracle.c (liboracle.so) of the reference's
  CPU adjacency-list algorithms, over CSR arrays.
* ``Ref``: the reference's own CPU algorithms compiled from its sources
  (oracle/_ref/libref.so, built by oracle/Makefile) behind a small C shim.

Only the tests, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline legs use
this package; the product (graphhet_b200) never imports it.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass
from typing import Optional

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
PORT_PATH = os.path.join(_HERE, "liboracle.so")
REF_PATH = os.path.join(_HERE, "_ref", "libref.so")

INT32_MAX = 2**31 - 1
DBL_MAX = 1.7976931348623157e308

_p = ctypes.c_void_p
_i32, _i64, _u64, _f64 = ctypes.c_int32, ctypes.c_int64, ctypes.c_uint64, ctypes.c_double

_port = None
_ref = None


def _np_ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_p)


def port() -> ctypes.CDLL:
    global _port
    if _port is None:
        if not os.path.exists(PORT_PATH):
            raise RuntimeError(f"{PORT_PATH} missing: run `make -C oracle`")
        L = ctypes.CDLL(PORT_PATH)
        sig = {
            "orc_gen_rmat": (None, [ctypes.c_int, _i64, _u64, _f64, _f64, _f64, ctypes.c_int, _p, _p]),
            "orc_gen_grid": (None, [_i32, _i32, _p, _p]),
            "orc_gen_er": (None, [_i32, _i64, _u64, _p, _p]),
            "orc_gen_dangling_keep": (None, [_i64, _p, _u64, ctypes.c_double, _p]),
            "orc_pair_weight": (_f64, [_u64, _i32, _i32, ctypes.c_int]),
            "orc_csr_build": (_i64, [_i32, _p, _p, _p, _i64, ctypes.c_int, ctypes.c_int, _u64, _p, _p, _p]),
            "orc_bfs": (None, [_i32, _p, _p, _i32, _i32, _p]),
            "orc_sssp": (None, [_i32, _p, _p, _p, _i32, _p]),
            "orc_wcc": (None, [_i32, _p, _p, _p]),
            "orc_pagerank": (None, [_i32, _p, _p, _p, _f64, _i32, _p]),
            "orc_cdlp": (None, [_i32, _p, _p, _p, _p, _i32, _p]),
            "orc_tc": (None, [_i32, _p, _p, _p]),
            "orc_tc_oriented": (_i64, [_i32, _p, _p, _p]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _port = L
    return _port


def ref_available() -> bool:
    return os.path.exists(REF_PATH)


# ------------------------------------------------------------------ inputs
def rmat_edges(scale: int, n_edges: int, seed: int, a=0.57, b=0.19, c=0.19, permute=True):
    src = np.empty(max(1, n_edges), np.int32)
    dst = np.empty(max(1, n_edges), np.int32)
    port().orc_gen_rmat(scale, n_edges, seed, a, b, c, int(permute), _np_ptr(src), _np_ptr(dst))
    return src[:n_edges], dst[:n_edges]


def grid_edges(rows: int, cols: int):
    ne = rows * (cols - 1) + (rows - 1) * cols
    src = np.empty(max(1, ne), np.int32)
    dst = np.empty(max(1, ne), np.int32)
    port().orc_gen_grid(rows, cols, _np_ptr(src), _np_ptr(dst))
    return src[:ne], dst[:ne]


def er_edges(n: int, n_edges: int, seed: int):
    src = np.empty(max(1, n_edges), np.int32)
    dst = np.empty(max(1, n_edges), np.int32)
    port().orc_gen_er(n, n_edges, seed, _np_ptr(src), _np_ptr(dst))
    return src[:n_edges], dst[:n_edges]


def dangling_keep(src, seed: int, fraction: float):
    src = np.ascontiguousarray(src, np.int32)
    keep = np.empty(max(1, src.size), np.uint8)
    port().orc_gen_dangling_keep(src.size, _np_ptr(src), seed, fraction, _np_ptr(keep))
    return keep[: src.size]


def build_csr(n, src, dst, w=None, symmetrize=False, drop_self_loops=True, transpose=False,
              weight_mode=1, weight_seed=0):
    src = np.ascontiguousarray(src, np.int32)
    dst = np.ascontiguousarray(dst, np.int32)
    ne = len(src)
    cap = max(1, ne * (2 if symmetrize else 1))
    rowptr = np.empty(n + 1, np.int32)
    col = np.empty(cap, np.int32)
    want_w = w is not None or weight_mode != 0
    wout = np.empty(cap, np.float64) if want_w else None
    flags = (1 if symmetrize else 0) | (2 if drop_self_loops else 0) | (4 if transpose else 0)
    win = np.ascontiguousarray(w, np.float64) if w is not None else None
    m = port().orc_csr_build(n, _np_ptr(src), _np_ptr(dst), _np_ptr(win), ne, flags, weight_mode, weight_seed,
                             _np_ptr(rowptr), _np_ptr(col), _np_ptr(wout))
    if m < 0:
        raise ValueError("edge endpoint outside [0, n)")
    return rowptr, col[:m].copy(), (wout[:m].copy() if wout is not None else None)


@dataclass
class Graph:
    """Host CSR (out and in) with the reference's layout."""
    n: int
    rowptr: np.ndarray
    col: np.ndarray
    w: Optional[np.ndarray]
    directed: bool
    in_rowptr: np.ndarray
    in_col: np.ndarray
    in_w: Optional[np.ndarray]

    @property
    def m(self):
        return len(self.col)


def make_graph(n, src, dst, directed, weight_mode=1, weight_seed=0, w=None) -> Graph:
    rp, col, wt = build_csr(n, src, dst, w=w, symmetrize=not directed, weight_mode=weight_mode,
                            weight_seed=weight_seed)
    if directed:
        irp, icol, iw = build_csr(n, src, dst, w=w, symmetrize=False, transpose=True, weight_mode=weight_mode,
                                  weight_seed=weight_seed)
    else:
        irp, icol, iw = rp, col, wt
    return Graph(n, rp, col, wt, directed, irp, icol, iw)


def rmat_graph(scale, edge_factor, seed, directed=False, a=0.57, b=0.19, c=0.19, weight_mode=1) -> Graph:
    src, dst = rmat_edges(scale, edge_factor << scale, seed, a, b, c, True)
    return make_graph(1 << scale, src, dst, directed, weight_mode=weight_mode, weight_seed=seed)


def grid_graph(rows, cols, weight_seed=0) -> Graph:
    src, dst = grid_edges(rows, cols)
    return make_graph(rows * cols, src, dst, False, weight_mode=2, weight_seed=weight_seed)


# ------------------------------------------------------- the C restatement
def bfs(g: Graph, src: int, max_depth: int = INT32_MAX):
    d = np.empty(g.n, np.int32)
    port().orc_bfs(g.n, _np_ptr(g.rowptr), _np_ptr(g.col), src, max_depth, _np_ptr(d))
    return d


def sssp(g: Graph, src: int):
    d = np.empty(g.n, np.float64)
    port().orc_sssp(g.n, _np_ptr(g.rowptr), _np_ptr(g.col), _np_ptr(g.w), src, _np_ptr(d))
    return d


def wcc(g: Graph):
    c = np.empty(g.n, np.int32)
    port().orc_wcc(g.n, _np_ptr(g.rowptr), _np_ptr(g.col), _np_ptr(c))
    return c


def pagerank(g: Graph, iterations=10, damping=0.85):
    r = np.empty(g.n, np.float64)
    port().orc_pagerank(g.n, _np_ptr(g.in_rowptr), _np_ptr(g.in_col), _np_ptr(g.rowptr), damping, iterations,
                        _np_ptr(r))
    return r


def cdlp(g: Graph, iterations=10):
    lab = np.empty(g.n, np.int32)
    port().orc_cdlp(g.n, _np_ptr(g.in_rowptr), _np_ptr(g.in_col), _np_ptr(g.rowptr), _np_ptr(g.col), iterations,
                    _np_ptr(lab))
    return lab


def tc(g: Graph):
    c = np.empty(g.n, np.int32)
    port().orc_tc(g.n, _np_ptr(g.rowptr), _np_ptr(g.col), _np_ptr(c))
    return c


def tc_oriented(g: Graph):
    """Per-vertex 6x triangle counts (int64, exact) and the triangle total by
    degree orientation, on all host threads: the checker for graphs where
    the reference's quadratic merge (tc above) does not finish.  Needs a
    symmetric, loop-free CSR without repeated entries."""
    c = np.empty(g.n, np.int64)
    t = port().orc_tc_oriented(g.n, _np_ptr(g.rowptr), _np_ptr(g.col), _np_ptr(c))
    return c, int(t)


# ------------------------------------------------------- dynamic graph
def gpma_keys(src, dst) -> np.ndarray:
    """KEY_TYPE (row << 32) | col (LDBC_GPU_gpma.cu:91-93) as int64."""
    return (np.asarray(src, np.int64) << 32) | np.asarray(dst, np.int64)


def gpma_update(keys: np.ndarray, vals: np.ndarray, bkeys, bvals):
    """One update_gpma batch (GPU_gpma.hpp:756-824) on a graph held as sorted
    unique int64 keys with their weights: for the last occurrence of every
    batch key, value 0 removes a present key (handle_del_mod,
    GPU_gpma.hpp:166-180), any other value overwrites a present key's weight
    or inserts the key.  Returns the new (keys, vals) and the counts
    (inserted, deleted, modified, ignored)."""
    bkeys = np.asarray(bkeys, np.int64)
    bvals = np.asarray(bvals, np.float64)
    order = np.argsort(bkeys, kind="stable")
    sk, sv = bkeys[order], bvals[order]
    last = np.ones(len(sk), bool)
    last[:-1] = sk[1:] != sk[:-1]
    uk, uv = sk[last], sv[last]
    pos = np.searchsorted(keys, uk)
    found = pos < len(keys)
    found[found] = keys[pos[found]] == uk[found]
    vals = vals.copy()
    mod = found & (uv != 0)
    vals[pos[mod]] = uv[mod]
    keep = np.ones(len(keys), bool)
    dele = found & (uv == 0)
    keep[pos[dele]] = False
    ins = ~found & (uv != 0)
    nk = np.concatenate([keys[keep], uk[ins]])
    nv = np.concatenate([vals[keep], uv[ins]])
    o = np.argsort(nk, kind="stable")
    counts = (int(ins.sum()), int(dele.sum()), int(mod.sum()), len(bkeys) - int(ins.sum() + dele.sum() + mod.sum()))
    return nk[o], nv[o], counts


def gpma_update_sequential(state: dict, bkeys, bvals) -> dict:
    """The same batch applied one update at a time, in batch order (small
    cases; pins gpma_update)."""
    for k, v in zip(np.asarray(bkeys, np.int64).tolist(), np.asarray(bvals, np.float64).tolist()):
        if v == 0.0:
            state.pop(k, None)
        else:
            state[k] = v
    return state


def gpma_from_csr(rowptr, col, w=None):
    rowptr = np.asarray(rowptr, np.int64)
    rows = np.repeat(np.arange(len(rowptr) - 1, dtype=np.int64), np.diff(rowptr))
    keys = gpma_keys(rows, col)
    vals = np.ones(len(keys)) if w is None else np.asarray(w, np.float64).copy()
    return keys, vals


def gpma_to_csr(n: int, keys: np.ndarray, vals: np.ndarray):
    rows = (keys >> 32).astype(np.int64)
    rowptr = np.zeros(n + 1, np.int32)
    np.add.at(rowptr, rows + 1, 1)
    return np.cumsum(rowptr).astype(np.int32), (keys & 0xFFFFFFFF).astype(np.int32), vals.copy()


# ------------------------------------------------- the reference, compiled
class Ref:
    """The reference's CPU algorithms (oracle/_ref/libref.so) on one loaded graph."""

    def __init__(self):
        if not ref_available():
            raise RuntimeError(f"{REF_PATH} missing: build with `make -C oracle` where the reference tree exists")
        L = ctypes.CDLL(REF_PATH)
        sig = {
            "ref_load": (ctypes.c_int, [ctypes.c_int, _p, _p, _p, _p, _p, _p]),
            "ref_free": (None, []),
            "ref_bfs": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _p]),
            "ref_bfs_pre": (ctypes.c_int, [ctypes.c_int, _p, _p]),
            "ref_sssp": (ctypes.c_int, [ctypes.c_int, _p]),
            "ref_sssp_pre": (ctypes.c_int, [ctypes.c_int, _p, _p]),
            "ref_wcc": (ctypes.c_int, [_p]),
            "ref_pagerank": (ctypes.c_int, [_f64, ctypes.c_int, _p]),
            "ref_cdlp": (ctypes.c_int, [ctypes.c_int, _p]),
            "ref_tc": (ctypes.c_int, [_p]),
            "ref_hardware_threads": (ctypes.c_int, []),
            "ref_apply_updates": (ctypes.c_int, [ctypes.c_longlong, _p, _p, _p]),
            "ref_out_entries": (ctypes.c_longlong, []),
            "ref_export_out": (ctypes.c_int, [_p, _p, _p]),
        }
        for k, (r, a) in sig.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        self.L = L
        self.n = 0

    def load(self, g: Graph):
        self._keep = g
        self.L.ref_load(g.n, _np_ptr(g.rowptr), _np_ptr(g.col), _np_ptr(g.w), _np_ptr(g.in_rowptr),
                        _np_ptr(g.in_col), _np_ptr(g.in_w))
        self.n = g.n
        return self

    def bfs(self, src, max_depth=INT32_MAX):
        d = np.empty(self.n, np.int32)
        self.L.ref_bfs(src, max_depth, _np_ptr(d))
        return d

    def bfs_pre(self, src):
        d = np.empty(self.n, np.int32)
        p = np.empty(self.n, np.int32)
        self.L.ref_bfs_pre(src, _np_ptr(d), _np_ptr(p))
        return d, p

    def sssp(self, src):
        d = np.empty(self.n, np.float64)
        self.L.ref_sssp(src, _np_ptr(d))
        return d

    def sssp_pre(self, src):
        d = np.empty(self.n, np.float64)
        p = np.empty(self.n, np.int32)
        self.L.ref_sssp_pre(src, _np_ptr(d), _np_ptr(p))
        return d, p

    def wcc(self):
        c = np.empty(self.n, np.int32)
        self.L.ref_wcc(_np_ptr(c))
        return c

    def pagerank(self, iterations=10, damping=0.85):
        r = np.empty(self.n, np.float64)
        self.L.ref_pagerank(damping, iterations, _np_ptr(r))
        return r

    def cdlp(self, iterations=10):
        lab = np.empty(self.n, np.int32)
        self.L.ref_cdlp(iterations, _np_ptr(lab))
        return lab

    def tc(self):
        c = np.empty(self.n, np.int32)
        self.L.ref_tc(_np_ptr(c))
        return c

    def apply_updates(self, src, dst, w):
        """Edits in order through graph_structure::add_edge / remove_edge."""
        src = np.ascontiguousarray(src, np.int32)
        dst = np.ascontiguousarray(dst, np.int32)
        w = np.ascontiguousarray(w, np.float64)
        self.L.ref_apply_updates(len(src), _np_ptr(src), _np_ptr(dst), _np_ptr(w))

    def export_out(self):
        m = int(self.L.ref_out_entries())
        rp = np.empty(self.n + 1, np.int32)
        col = np.empty(max(1, m), np.int32)
        w = np.empty(max(1, m), np.float64)
        self.L.ref_export_out(_np_ptr(rp), _np_ptr(col), _np_ptr(w))
        return rp, col[:m], w[:m]

    def hardware_threads(self):
        return int(self.L.ref_hardware_threads())

    def close(self):
        self.L.ref_free()
