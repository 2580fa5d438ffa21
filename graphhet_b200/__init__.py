"""graphhet_b200: GraphHET's CSR analytics path (BFS, SSSP, WCC, PageRank,
CDLP, triangle counting) on B200 (sm_100a).

The compute lives in ``libghb.so`` (hand-written CUDA behind the C ABI of
``include/ghb.h``).  This module is a thin host layer over that ABI: torch
tensors hold the device memory, ctypes passes their pointers.  There is no
CPU fallback: if the library is missing every call raises.

Entry points mirror the reference's (include/GPU_csr/algorithm/*.cuh):
``bfs`` ~ Cuda_BFS, ``sssp`` ~ Cuda_SSSP, ``wcc`` ~ Cuda_WCC,
``pagerank`` ~ Cuda_PR, ``cdlp`` ~ Cuda_CDLP, ``tc`` ~ Cuda_TC, and
``bfs_pred`` / ``sssp_pred`` ~ Cuda_BFS_pre / Cuda_SSSP_pre.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass, field
from typing import Optional

import torch

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libghb.so")

INT32_MAX = 2**31 - 1
DBL_MAX = 1.7976931348623157e308

POLICY_HEURISTIC, POLICY_LEARNED, POLICY_PUSH, POLICY_PULL, POLICY_SCHEDULE = 0, 1, 2, 3, 4
PR_FP64, PR_FP32_KAHAN = 0, 1
BUILD_SYMMETRIZE, BUILD_DROP_SELF_LOOPS, BUILD_TRANSPOSE = 1, 2, 4
WEIGHT_NONE, WEIGHT_UNIFORM01, WEIGHT_INT100 = 0, 1, 2
TRACE_FEATURES, TRACE_COLS = 12, 24
POLICY_PARAMS, POLICY_OUT = 6292, 20

_p = ctypes.c_void_p
_i32 = ctypes.c_int32
_i64 = ctypes.c_int64
_u64 = ctypes.c_uint64
_f64 = ctypes.c_double


class BfsOptions(ctypes.Structure):
    _fields_ = [("policy", _i32), ("alpha", ctypes.c_float), ("beta", ctypes.c_float),
                ("schedule", _p), ("schedule_len", _i32), ("record_trace", _i32),
                ("trace", _p), ("trace_cap", _i32), ("oracle_timing", _i32), ("gamma", ctypes.c_float)]


class SsspOptions(ctypes.Structure):
    _fields_ = [("delta", _f64), ("policy", _i32), ("record_trace", _i32), ("trace", _p),
                ("trace_cap", _i32)]


class TraversalStats(ctypes.Structure):
    _fields_ = [("levels", _i32), ("pull_levels", _i32), ("reached", _i64),
                ("edges_reached", _i64), ("edges_examined", _i64), ("device_ms", _f64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class MsbfsOptions(ctypes.Structure):
    _fields_ = [("schedule", _p), ("schedule_len", _i32), ("trace", _p), ("trace_cap", _i32)]


MS_TRACE_COLS = 6


class PrOptions(ctypes.Structure):
    _fields_ = [("iterations", _i32), ("damping", _f64), ("precision", _i32),
                ("tolerance", _f64), ("l1_history", _p)]


# name -> (restype, argtypes)
_SIGS = {
    "ghb_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "ghb_last_error": (ctypes.c_char_p, []),
    "ghb_version": (ctypes.c_int, []),
    "ghb_workspace_create": (ctypes.c_int, [ctypes.POINTER(_p)]),
    "ghb_workspace_destroy": (ctypes.c_int, [_p]),
    "ghb_workspace_set_stream": (ctypes.c_int, [_p, _p]),
    "ghb_workspace_get_stream": (_p, [_p]),
    "ghb_workspace_trim": (ctypes.c_int, [_p]),
    "ghb_workspace_counters": (ctypes.c_int, [_p, ctypes.POINTER(_i64), ctypes.POINTER(_i64)]),
    "ghb_default_workspace": (_p, []),
    "ghb_tune_set": (ctypes.c_int, [_p, ctypes.c_char_p, _i32]),
    "ghb_tune_get": (ctypes.c_int, [_p, ctypes.c_char_p, ctypes.POINTER(_i32)]),
    "ghb_gen_rmat": (ctypes.c_int, [_p, _i32, _i64, _u64, _f64, _f64, _f64, _i32, _p, _p]),
    "ghb_gen_grid": (ctypes.c_int, [_p, _i32, _i32, _p, _p]),
    "ghb_gen_er": (ctypes.c_int, [_p, _i32, _i64, _u64, _p, _p]),
    "ghb_gen_powerlaw": (ctypes.c_int, [_p, _i32, _i64, _f64, _u64, _p, _p]),
    "ghb_gen_dangling_keep": (ctypes.c_int, [_p, _i64, _p, _u64, _f64, _p]),
    "ghb_csr_build": (ctypes.c_int, [_p, _i32, _p, _p, _p, _i64, _i32, _i32, _u64, _p, _p, _p,
                                     ctypes.POINTER(_i64)]),
    "ghb_csr_transpose": (ctypes.c_int, [_p, _i32, _i64, _p, _p, _p, _p, _p, _p]),
    "ghb_csr_merge_in_out": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p, _p]),
    "ghb_bfs": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _i32, _i32, _p, _p, _p]),
    "ghb_bfs_pred": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _i32, _i32, _p, _p, _p, _p]),
    "ghb_msbfs": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p, _i32, _p, _p]),
    "ghb_sssp": (ctypes.c_int, [_p, _i32, _p, _p, _p, _i32, _f64, _p, _p, _p]),
    "ghb_sssp_pred": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p, _p, _i32, _f64, _p, _p, _p, _p]),
    "ghb_mssssp": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _i32, _f64, _p, _p]),
    "ghb_wcc": (ctypes.c_int, [_p, _i32, _p, _p, _p]),
    "ghb_pagerank": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p, _p]),
    "ghb_cdlp": (ctypes.c_int, [_p, _i32, _p, _p, _i32, _p]),
    "ghb_tc": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p]),
    "ghb_batch_wcc": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p]),
    "ghb_batch_tc": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p, _p]),
    "ghb_union_reserve": (ctypes.c_int, [_p, _i32, _i64]),
    "ghb_ldbc_load": (ctypes.c_int, [_p, ctypes.c_char_p, ctypes.c_char_p, _i32, ctypes.POINTER(_p)]),
    "ghb_ldbc_info": (ctypes.c_int, [_p, ctypes.POINTER(_i32), ctypes.POINTER(_i64), ctypes.POINTER(_i32)]),
    "ghb_ldbc_csr": (ctypes.c_int, [_p] + [ctypes.POINTER(_p)] * 6),
    "ghb_ldbc_copy": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _p, _p]),
    "ghb_ldbc_name": (ctypes.c_int, [_p, _i32, ctypes.POINTER(ctypes.c_char_p)]),
    "ghb_ldbc_id": (ctypes.c_int, [_p, ctypes.c_char_p, ctypes.POINTER(_i32)]),
    "ghb_ldbc_free": (ctypes.c_int, [_p]),
    "ghb_union_wcc_tc": (ctypes.c_int, [_p, _i32, _p, _i32, _i64, _p, _p, _p, _p, _p]),
    "ghb_graph_create": (ctypes.c_int, [_p, _i32, _p, _p, _p, _p, _p, _p, ctypes.POINTER(_p)]),
    "ghb_graph_destroy": (ctypes.c_int, [_p]),
    "ghb_graph_info": (ctypes.c_int, [_p, ctypes.POINTER(_i64), ctypes.POINTER(_i32), ctypes.POINTER(_i64),
                                      ctypes.POINTER(ctypes.c_float)]),
    "ghb_graph_perm": (ctypes.c_int, [_p, ctypes.POINTER(_p), ctypes.POINTER(_p)]),
    "ghb_graph_bfs": (ctypes.c_int, [_p, _p, _i32, _i32, _p, _p, _p]),
    "ghb_graph_bfs_pred": (ctypes.c_int, [_p, _p, _i32, _i32, _p, _p, _p, _p]),
    "ghb_graph_bfs_many_host": (ctypes.c_int, [_p, _p, _p, _i32, _i32, _p, _i32, _p, _p]),
    "ghb_graph_msbfs_ex": (ctypes.c_int, [_p, _p, _p, _i32, _p, _p, _p]),
    "ghb_ms_policy_load": (ctypes.c_int, [_p, _i32]),
    "ghb_graph_msbfs": (ctypes.c_int, [_p, _p, _p, _i32, _p, _p]),
    "ghb_graph_msbfs_reserve": (ctypes.c_int, [_p, _p, _i32]),
    "ghb_graph_msbfs_launch": (ctypes.c_int, [_p, _p, _p, _i32, _p]),
    "ghb_graph_sssp": (ctypes.c_int, [_p, _p, _i32, _f64, _p, _p, _p]),
    "ghb_graph_mssssp": (ctypes.c_int, [_p, _p, _p, _i32, _f64, _p, _p]),
    "ghb_graph_sssp_pred": (ctypes.c_int, [_p, _p, _i32, _f64, _p, _p, _p, _p]),
    "ghb_graph_wcc": (ctypes.c_int, [_p, _p, _p]),
    "ghb_graph_pagerank": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "ghb_graph_cdlp": (ctypes.c_int, [_p, _p, _i32, _p]),
    "ghb_graph_tc": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "ghb_policy_load": (ctypes.c_int, [_p, _p]),
    "ghb_policy_loaded": (ctypes.c_int, []),
    "ghb_mlp_forward": (ctypes.c_int, [_p, _p, _p, _p, _i32, _p]),
    "ghb_mlp_grad": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _i32, _p, ctypes.POINTER(ctypes.c_float)]),
    "ghb_mlp_train": (ctypes.c_int, [_p, _p, _p, _p, _p, _p, _i32, _i32, ctypes.c_float, _p]),
    "ghb_gpma_create": (ctypes.c_int, [_p, _i32, ctypes.POINTER(_p)]),
    "ghb_gpma_destroy": (ctypes.c_int, [_p]),
    "ghb_gpma_clone": (ctypes.c_int, [_p, _p, ctypes.POINTER(_p)]),
    "ghb_gpma_clear": (ctypes.c_int, [_p, _p]),
    "ghb_gpma_load_csr": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "ghb_gpma_update": (ctypes.c_int, [_p, _p, _p, _p, _i64, _p]),
    "ghb_gpma_info": (ctypes.c_int, [_p, ctypes.POINTER(_i32), ctypes.POINTER(_i64), ctypes.POINTER(_i64),
                                     ctypes.POINTER(_i64)]),
    "ghb_gpma_stats": (ctypes.c_int, [_p, _p]),
    "ghb_gpma_csr": (ctypes.c_int, [_p, _p, _i32, ctypes.POINTER(_p), ctypes.POINTER(_p), ctypes.POINTER(_p)]),
    "ghb_gpma_export": (ctypes.c_int, [_p, _p, _p, _p, _p]),
    "ghb_gpma_find": (ctypes.c_int, [_p, _p, _p, _i64, _p]),
}

_lib = None


class GhbError(RuntimeError):
    pass


def lib() -> ctypes.CDLL:
    """Load libghb.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise GhbError(f"{LIB_PATH} is missing: build it with `make` (or __graft_entry__.build())")
        L = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGS.items():
            fn = getattr(L, name, None)
            if fn is None:
                continue
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(status: int, what: str) -> None:
    if status != 0:
        L = lib()
        raise GhbError(f"{what}: {L.ghb_status_string(status).decode()} "
                       f"({L.ghb_last_error().decode()})")


def _ptr(t: Optional[torch.Tensor]):
    if t is None:
        return None
    if not t.is_cuda:
        raise GhbError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise GhbError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


class Workspace:
    """A libghb workspace bound to torch's current CUDA stream."""

    def __init__(self):
        self._h = _p()
        _check(lib().ghb_workspace_create(ctypes.byref(self._h)), "ghb_workspace_create")

    @property
    def handle(self):
        lib().ghb_workspace_set_stream(self._h, _p(torch.cuda.current_stream().cuda_stream))
        return self._h

    def counters(self):
        launches, scratch = _i64(), _i64()
        _check(lib().ghb_workspace_counters(self._h, ctypes.byref(launches), ctypes.byref(scratch)),
               "ghb_workspace_counters")
        return launches.value, scratch.value

    def trim(self):
        _check(lib().ghb_workspace_trim(self._h), "ghb_workspace_trim")

    def close(self):
        if self._h:
            lib().ghb_workspace_destroy(self._h)
            self._h = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


TUNABLES = ("pr_cache_kb", "pr_threads", "pr_blocks_per_sm", "pr_short", "pr_chunk", "ms_warp_rest", "ms_pull_div",
            "pol_band")


def tune_set(name: str, value: int, ws=None) -> None:
    """Set a launch shape / threshold of the workspace (results do not change)."""
    _check(lib().ghb_tune_set(_ws(ws), name.encode(), int(value)), "ghb_tune_set")


def tune_get(name: str, ws=None) -> int:
    v = _i32()
    _check(lib().ghb_tune_get(_ws(ws), name.encode(), ctypes.byref(v)), "ghb_tune_get")
    return v.value


_default_ws: dict = {}


def default_workspace() -> Workspace:
    dev = torch.cuda.current_device()
    ws = _default_ws.get(dev)
    if ws is None:
        ws = _default_ws[dev] = Workspace()
    return ws


def _ws(ws):
    return (ws or default_workspace()).handle


# --------------------------------------------------------------- graphs
@dataclass
class CSRGraph:
    """Device CSR in the reference's layout (CSR_graph, GPU_csr.hpp:97-110).

    For an undirected graph the in/all arrays are the out arrays, as toCSR
    aliases them (GPU_csr.hpp:133-140)."""
    n: int
    rowptr: torch.Tensor
    col: torch.Tensor
    w: Optional[torch.Tensor] = None
    directed: bool = False
    in_rowptr: Optional[torch.Tensor] = None
    in_col: Optional[torch.Tensor] = None
    in_w: Optional[torch.Tensor] = None
    _all: Optional[tuple] = field(default=None, repr=False)

    @property
    def m(self) -> int:
        return int(self.col.numel())

    def in_csr(self):
        if not self.directed:
            return self.rowptr, self.col, self.w
        return self.in_rowptr, self.in_col, self.in_w

    def all_csr(self, ws=None):
        """Row v = in-neighbours then out-neighbours (toCSR, GPU_csr.hpp:315-330)."""
        if not self.directed:
            return self.rowptr, self.col
        if self._all is None:
            arp = torch.empty(self.n + 1, dtype=torch.int32, device=self.rowptr.device)
            acol = torch.empty(max(1, self.m + int(self.in_col.numel())), dtype=torch.int32,
                               device=self.rowptr.device)
            _check(lib().ghb_csr_merge_in_out(_ws(ws), self.n, _ptr(self.in_rowptr), _ptr(self.in_col),
                                              _ptr(self.rowptr), _ptr(self.col), _ptr(arp), _ptr(acol)),
                   "ghb_csr_merge_in_out")
            self._all = (arp, acol[: self.m + int(self.in_col.numel())])
        return self._all


def _dev(device):
    return torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())


def gen_rmat(scale: int, n_edges: int, seed: int, a=0.57, b=0.19, c=0.19, permute=True, device=None, ws=None):
    d = _dev(device)
    src = torch.empty(max(1, n_edges), dtype=torch.int32, device=d)
    dst = torch.empty(max(1, n_edges), dtype=torch.int32, device=d)
    _check(lib().ghb_gen_rmat(_ws(ws), scale, n_edges, seed, a, b, c, int(permute), _ptr(src), _ptr(dst)),
           "ghb_gen_rmat")
    return src[:n_edges], dst[:n_edges]


def gen_grid(rows: int, cols: int, device=None, ws=None):
    d = _dev(device)
    ne = rows * (cols - 1) + (rows - 1) * cols
    src = torch.empty(max(1, ne), dtype=torch.int32, device=d)
    dst = torch.empty(max(1, ne), dtype=torch.int32, device=d)
    _check(lib().ghb_gen_grid(_ws(ws), rows, cols, _ptr(src), _ptr(dst)), "ghb_gen_grid")
    return src[:ne], dst[:ne]


def gen_er(n: int, n_edges: int, seed: int, device=None, ws=None):
    d = _dev(device)
    src = torch.empty(max(1, n_edges), dtype=torch.int32, device=d)
    dst = torch.empty(max(1, n_edges), dtype=torch.int32, device=d)
    _check(lib().ghb_gen_er(_ws(ws), n, n_edges, seed, _ptr(src), _ptr(dst)), "ghb_gen_er")
    return src[:n_edges], dst[:n_edges]


def gen_powerlaw(scale: int, n_edges: int, exponent: float, seed: int, device=None, ws=None):
    dev = _dev(device)
    src = torch.empty(n_edges, dtype=torch.int32, device=dev)
    dst = torch.empty(n_edges, dtype=torch.int32, device=dev)
    _check(lib().ghb_gen_powerlaw(_ws(ws), scale, n_edges, exponent, seed, _ptr(src), _ptr(dst)),
           "ghb_gen_powerlaw")
    return src, dst


def build_csr(n: int, src: torch.Tensor, dst: torch.Tensor, w: Optional[torch.Tensor] = None,
              symmetrize=False, drop_self_loops=True, transpose=False, weight_mode=WEIGHT_UNIFORM01,
              weight_seed=0, ws=None):
    """Edge list -> (rowptr, col, w) with sorted, deduplicated rows (ghb_csr_build)."""
    ne = int(src.numel())
    cap = max(1, ne * (2 if symmetrize else 1))
    dev = src.device
    rowptr = torch.empty(n + 1, dtype=torch.int32, device=dev)
    col = torch.empty(cap, dtype=torch.int32, device=dev)
    want_w = w is not None or weight_mode != WEIGHT_NONE
    wout = torch.empty(cap, dtype=torch.float64, device=dev) if want_w else None
    flags = (BUILD_SYMMETRIZE if symmetrize else 0) | (BUILD_DROP_SELF_LOOPS if drop_self_loops else 0) | \
            (BUILD_TRANSPOSE if transpose else 0)
    m = _i64()
    _check(lib().ghb_csr_build(_ws(ws), n, _ptr(src.contiguous()), _ptr(dst.contiguous()),
                               _ptr(w.contiguous()) if w is not None else None, ne, flags, weight_mode,
                               weight_seed, _ptr(rowptr), _ptr(col), _ptr(wout), ctypes.byref(m)),
           "ghb_csr_build")
    mm = m.value
    # Shrink to the entry count (frees the worst-case allocation).
    col = col[:mm].clone()
    wout = wout[:mm].clone() if wout is not None else None
    return rowptr, col, wout


def transpose_csr(n: int, rowptr, col, w=None, ws=None):
    m = int(col.numel())
    trp = torch.empty(n + 1, dtype=torch.int32, device=rowptr.device)
    tcol = torch.empty(max(1, m), dtype=torch.int32, device=rowptr.device)
    tw = torch.empty(max(1, m), dtype=torch.float64, device=rowptr.device) if w is not None else None
    _check(lib().ghb_csr_transpose(_ws(ws), n, m, _ptr(rowptr), _ptr(col) if m else None,
                                   _ptr(w) if (w is not None and m) else None, _ptr(trp), _ptr(tcol),
                                   _ptr(tw) if tw is not None else None), "ghb_csr_transpose")
    return trp, tcol[:m], (tw[:m] if tw is not None else None)


def make_graph(n: int, src, dst, directed: bool, weight_mode=WEIGHT_UNIFORM01, weight_seed=0, w=None,
               drop_self_loops=True, ws=None) -> CSRGraph:
    rp, col, wt = build_csr(n, src, dst, w=w, symmetrize=not directed, drop_self_loops=drop_self_loops,
                            weight_mode=weight_mode, weight_seed=weight_seed, ws=ws)
    g = CSRGraph(n=n, rowptr=rp, col=col, w=wt, directed=directed)
    if directed:
        g.in_rowptr, g.in_col, g.in_w = transpose_csr(n, rp, col, wt, ws=ws)
    return g


def rmat_graph(scale: int, edge_factor: int, seed: int, directed=False, a=0.57, b=0.19, c=0.19,
               weight_mode=WEIGHT_UNIFORM01, device=None, ws=None) -> CSRGraph:
    """RMAT(scale, edge_factor) with permuted ids, duplicates and self-loops removed."""
    src, dst = gen_rmat(scale, edge_factor << scale, seed, a, b, c, True, device=device, ws=ws)
    g = make_graph(1 << scale, src, dst, directed, weight_mode=weight_mode, weight_seed=seed, ws=ws)
    del src, dst
    return g


def rmat_dangling_graph(scale: int, edge_factor: int, seed: int, fraction: float = 0.1, device=None,
                        ws=None) -> CSRGraph:
    """Directed RMAT(scale, edge_factor) whose seeded `fraction` of vertices
    lose all out-edges (the PageRank precision workload), no weights."""
    src, dst = gen_rmat(scale, edge_factor << scale, seed, 0.57, 0.19, 0.19, True, device=device, ws=ws)
    keep = torch.empty(src.numel(), dtype=torch.uint8, device=src.device)
    _check(lib().ghb_gen_dangling_keep(_ws(ws), src.numel(), _ptr(src), seed, fraction, _ptr(keep)),
           "ghb_gen_dangling_keep")
    k = keep.bool()
    src, dst = src[k].contiguous(), dst[k].contiguous()
    del keep, k
    return make_graph(1 << scale, src, dst, True, weight_mode=WEIGHT_NONE, ws=ws)


def load_ldbc(vertex_path: str, edge_path: str, directed: bool, ws=None):
    """LDBC .v/.e files -> (CSRGraph on the device, vertex names by id).  The
    library parses them with every host thread and builds the CSR on the GPU
    (ghb_ldbc_load); the arrays are copied out of its handle."""
    h = _p()
    _check(lib().ghb_ldbc_load(_ws(ws), vertex_path.encode(), edge_path.encode(), int(directed), ctypes.byref(h)),
           "ghb_ldbc_load")
    try:
        n, m, wt = _i32(), _i64(), _i32()
        _check(lib().ghb_ldbc_info(h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(wt)), "ghb_ldbc_info")
        n, m = n.value, m.value
        t = lambda k, dt: torch.empty(max(1, k), dtype=dt, device="cuda")
        rp, col, w = t(n + 1, torch.int32), t(m, torch.int32), t(m, torch.float64)
        irp, icol, iw = (t(n + 1, torch.int32), t(m, torch.int32), t(m, torch.float64)) if directed else (None,) * 3
        _check(lib().ghb_ldbc_copy(_ws(ws), h, _ptr(rp), _ptr(col), _ptr(w), _ptr(irp), _ptr(icol), _ptr(iw)),
               "ghb_ldbc_copy")
        torch.cuda.synchronize()
        g = CSRGraph(n=n, rowptr=rp, col=col[:m], w=w[:m], directed=directed)
        if directed:
            g.in_rowptr, g.in_col, g.in_w = irp, icol[:m], iw[:m]
        names = []
        nm = ctypes.c_char_p()
        for i in range(n):
            _check(lib().ghb_ldbc_name(h, i, ctypes.byref(nm)), "ghb_ldbc_name")
            names.append(nm.value.decode())
        return g, names
    finally:
        lib().ghb_ldbc_free(h)


class UnionBatch:
    """Many independent graphs as one disjoint-union CSR (ghb_union_*): graph
    g owns global vertices [vbase[g], vbase[g+1])."""

    def __init__(self, vbase, g: CSRGraph):
        self.vbase = torch.as_tensor(vbase, dtype=torch.int64).to(g.rowptr.device)
        self.vbase_host = self.vbase.cpu().numpy()
        self.g = g
        self.n_graphs = len(self.vbase_host) - 1

    def reserve(self, ws=None):
        _check(lib().ghb_union_reserve(_ws(ws), self.g.n, self.g.m), "ghb_union_reserve")

    def wcc_tc(self, label=None, counts64=None, triangles=None, ws=None):
        """Fills the given device tensors (label int32[n_total], counts64
        int64[n_total], triangles int64[n_graphs]); launches only."""
        _check(lib().ghb_union_wcc_tc(_ws(ws), self.n_graphs, _ptr(self.vbase), self.g.n, self.g.m,
                                      _ptr(self.g.rowptr), _ptr(self.g.col) if self.g.m else None, _ptr(label),
                                      _ptr(counts64), _ptr(triangles)), "ghb_union_wcc_tc")


def er_batch(n_graphs: int, seed: int, n_lo: int = 1000, n_hi: int = 200000, deg_lo: float = 2.0,
             deg_hi: float = 32.0, device=None, ws=None) -> UnionBatch:
    """n_graphs Erdos-Renyi graphs, n log-uniform in [n_lo, n_hi], mean degree
    uniform in [deg_lo, deg_hi] (edges = n * degree / 2, ghb_gen_er with seed
    seed * 1000003 + g), symmetrised and deduplicated, as one union CSR."""
    import numpy as np
    rng = np.random.default_rng(seed)
    ns = np.exp(rng.uniform(np.log(n_lo), np.log(n_hi), n_graphs)).astype(np.int64)
    degs = rng.uniform(deg_lo, deg_hi, n_graphs)
    es = (ns * degs / 2).astype(np.int64)
    vbase = np.concatenate([[0], np.cumsum(ns)]).astype(np.int64)
    ebase = np.concatenate([[0], np.cumsum(es)]).astype(np.int64)
    d = _dev(device)
    src = torch.empty(int(ebase[-1]), dtype=torch.int32, device=d)
    dst = torch.empty(int(ebase[-1]), dtype=torch.int32, device=d)
    for gi in range(n_graphs):
        s, t = gen_er(int(ns[gi]), int(es[gi]), seed * 1000003 + gi, device=d, ws=ws)
        src[ebase[gi]:ebase[gi + 1]] = s + int(vbase[gi])
        dst[ebase[gi]:ebase[gi + 1]] = t + int(vbase[gi])
    g = make_graph(int(vbase[-1]), src, dst, False, weight_mode=WEIGHT_NONE, ws=ws)
    del src, dst
    return UnionBatch(vbase, g)


def grid_graph(rows: int, cols: int, weight_seed=0, device=None, ws=None) -> CSRGraph:
    """rows x cols 4-neighbour grid, integer weights in [1, 100]."""
    src, dst = gen_grid(rows, cols, device=device, ws=ws)
    return make_graph(rows * cols, src, dst, False, weight_mode=WEIGHT_INT100, weight_seed=weight_seed, ws=ws)


# ----------------------------------------------------------- algorithms
def _stats_out(stats: TraversalStats):
    return stats.as_dict()


def bfs(g: CSRGraph, src: int, max_depth: int = INT32_MAX, policy: int = POLICY_HEURISTIC, alpha=0.0,
        beta=0.0, schedule=None, trace_cap: int = 0, oracle_timing=False, out=None, ws=None):
    """Depths from src (INT32_MAX = unreached).  Returns (depth, stats[, trace])."""
    depth = out if out is not None else torch.empty(g.n, dtype=torch.int32, device=g.rowptr.device)
    irp, icol, _ = g.in_csr()
    opt = BfsOptions(policy=policy, alpha=alpha, beta=beta)
    sched_buf = None
    if schedule is not None:
        sched_buf = (ctypes.c_int8 * len(schedule))(*[int(x) for x in schedule])
        opt.schedule = ctypes.cast(sched_buf, _p)
        opt.schedule_len = len(schedule)
    trace = None
    if trace_cap > 0:
        trace = (ctypes.c_float * (trace_cap * TRACE_COLS))()
        opt.record_trace = 1
        opt.trace = ctypes.cast(trace, _p)
        opt.trace_cap = trace_cap
        opt.oracle_timing = int(oracle_timing)
    st = TraversalStats()
    _check(lib().ghb_bfs(_ws(ws), g.n, _ptr(g.rowptr), _ptr(g.col) if g.m else None, _ptr(irp),
                         _ptr(icol) if icol is not None and icol.numel() else None, src, max_depth,
                         _ptr(depth), ctypes.byref(opt), ctypes.byref(st)), "ghb_bfs")
    if trace is not None:
        import numpy as np
        rows = min(trace_cap, st.levels)
        tr = np.frombuffer(trace, dtype=np.float32).reshape(trace_cap, TRACE_COLS)[:rows].copy()
        return depth, _stats_out(st), tr
    return depth, _stats_out(st)


def bfs_pred(g: CSRGraph, src: int, max_depth: int = INT32_MAX, ws=None):
    depth = torch.empty(g.n, dtype=torch.int32, device=g.rowptr.device)
    pred = torch.empty(g.n, dtype=torch.int32, device=g.rowptr.device)
    irp, icol, _ = g.in_csr()
    st = TraversalStats()
    _check(lib().ghb_bfs_pred(_ws(ws), g.n, _ptr(g.rowptr), _ptr(g.col) if g.m else None, _ptr(irp),
                              _ptr(icol) if icol is not None and icol.numel() else None, src, max_depth,
                              _ptr(depth), _ptr(pred), None, ctypes.byref(st)), "ghb_bfs_pred")
    return depth, pred


def sssp(g: CSRGraph, src: int, inf: float = DBL_MAX, delta: float = 0.0, out=None, ws=None):
    """FP64 distances from src (`inf` = unreached).  Returns (dist, stats)."""
    dist = out if out is not None else torch.empty(g.n, dtype=torch.float64, device=g.rowptr.device)
    opt = SsspOptions(delta=delta)
    st = TraversalStats()
    _check(lib().ghb_sssp(_ws(ws), g.n, _ptr(g.rowptr), _ptr(g.col) if g.m else None,
                          _ptr(g.w) if g.m else None, src, inf, _ptr(dist), ctypes.byref(opt),
                          ctypes.byref(st)), "ghb_sssp")
    return dist, _stats_out(st)


def sssp_pred(g: CSRGraph, src: int, inf: float = DBL_MAX, ws=None):
    dist = torch.empty(g.n, dtype=torch.float64, device=g.rowptr.device)
    pred = torch.empty(g.n, dtype=torch.int32, device=g.rowptr.device)
    irp, icol, iw = g.in_csr()
    st = TraversalStats()
    has = g.m > 0
    _check(lib().ghb_sssp_pred(_ws(ws), g.n, _ptr(g.rowptr), _ptr(g.col) if has else None,
                               _ptr(g.w) if has else None, _ptr(irp), _ptr(icol) if has else None,
                               _ptr(iw) if has else None, src, inf, _ptr(dist), _ptr(pred), None,
                               ctypes.byref(st)), "ghb_sssp_pred")
    return dist, pred


def wcc(g: CSRGraph, out=None, ws=None):
    """Smallest vertex id of each vertex's weak component."""
    lab = out if out is not None else torch.empty(g.n, dtype=torch.int32, device=g.rowptr.device)
    _check(lib().ghb_wcc(_ws(ws), g.n, _ptr(g.rowptr), _ptr(g.col) if g.m else None, _ptr(lab)), "ghb_wcc")
    return lab


def pagerank(g: CSRGraph, iterations: int = 10, damping: float = 0.85, precision: int = PR_FP64,
             tolerance: float = 0.0, l1_history=False, out=None, ws=None):
    """LDBC PageRank.  Returns (rank, iterations_run, l1_per_iteration or None)."""
    rank = out if out is not None else torch.empty(g.n, dtype=torch.float64, device=g.rowptr.device)
    irp, icol, _ = g.in_csr()
    hist = (ctypes.c_double * max(1, iterations))() if l1_history else None
    opt = PrOptions(iterations=iterations, damping=damping, precision=precision, tolerance=tolerance,
                    l1_history=ctypes.cast(hist, _p) if hist is not None else None)
    ran = _i32()
    _check(lib().ghb_pagerank(_ws(ws), g.n, _ptr(irp), _ptr(icol) if icol.numel() else None, _ptr(g.rowptr),
                              ctypes.byref(opt), _ptr(rank), ctypes.byref(ran)), "ghb_pagerank")
    h = list(hist)[: ran.value] if hist is not None else None
    return rank, ran.value, h


def cdlp(g: CSRGraph, iterations: int = 10, out=None, ws=None):
    """Label propagation over in+out neighbours, smallest label on ties."""
    lab = out if out is not None else torch.empty(g.n, dtype=torch.int32, device=g.rowptr.device)
    arp, acol = g.all_csr(ws)
    _check(lib().ghb_cdlp(_ws(ws), g.n, _ptr(arp), _ptr(acol) if acol.numel() else None, iterations,
                          _ptr(lab)), "ghb_cdlp")
    return lab


def tc(g: CSRGraph, ws=None):
    """Per-vertex counts as the reference computes them.  Returns
    (counts64, counts32 (the reference's wrapping int32), triangles)."""
    c64 = torch.empty(g.n, dtype=torch.int64, device=g.rowptr.device)
    c32 = torch.empty(g.n, dtype=torch.int32, device=g.rowptr.device)
    total = _i64()
    _check(lib().ghb_tc(_ws(ws), g.n, _ptr(g.rowptr), _ptr(g.col) if g.m else None, _ptr(c64), _ptr(c32),
                        ctypes.byref(total)), "ghb_tc")
    return c64, c32, total.value


# ------------------------------------------------------- resident graphs
class ResidentGraph:
    """A graph relabelled once by degree on the GPU (ghb_graph_create); every
    method returns the same values as the module-level function of the same
    name, in the caller's vertex ids."""

    def __init__(self, g: CSRGraph, ws=None):
        self.n = g.n
        self.directed = g.directed
        self._dev = g.rowptr.device
        self._h = _p()
        irp, icol, iw = g.in_csr()
        has = g.m > 0
        _check(lib().ghb_graph_create(_ws(ws), g.n, _ptr(g.rowptr), _ptr(g.col) if has else None,
                                      _ptr(g.w) if (g.w is not None and has) else None,
                                      _ptr(irp) if g.directed else None,
                                      _ptr(icol) if (g.directed and icol.numel()) else None,
                                      _ptr(iw) if (g.directed and iw is not None and iw.numel()) else None,
                                      ctypes.byref(self._h)), "ghb_graph_create")
        m, na, nb, ms = _i64(), _i32(), _i64(), ctypes.c_float()
        _check(lib().ghb_graph_info(self._h, ctypes.byref(m), ctypes.byref(na), ctypes.byref(nb), ctypes.byref(ms)),
               "ghb_graph_info")
        self.m, self.n_active, self.device_bytes, self.build_ms = m.value, na.value, nb.value, ms.value

    def close(self):
        if self._h:
            lib().ghb_graph_destroy(self._h)
            self._h = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _i32(self, k=1):
        return torch.empty(self.n * k, dtype=torch.int32, device=self._dev)

    def bfs(self, src, max_depth=INT32_MAX, policy=POLICY_HEURISTIC, schedule=None, trace_cap=0,
            oracle_timing=False, alpha=0.0, beta=0.0, gamma=0.0, out=None, ws=None):
        depth = out if out is not None else self._i32()
        opt = BfsOptions(policy=policy, alpha=alpha, beta=beta, gamma=gamma)
        keep = None
        if schedule is not None:
            keep = (ctypes.c_int8 * len(schedule))(*[int(x) for x in schedule])
            opt.schedule = ctypes.cast(keep, _p)
            opt.schedule_len = len(schedule)
        trace = None
        if trace_cap > 0:
            trace = (ctypes.c_float * (trace_cap * TRACE_COLS))()
            opt.record_trace, opt.trace, opt.trace_cap = 1, ctypes.cast(trace, _p), trace_cap
            opt.oracle_timing = int(oracle_timing)
        st = TraversalStats()
        _check(lib().ghb_graph_bfs(_ws(ws), self._h, src, max_depth, _ptr(depth), ctypes.byref(opt),
                                   ctypes.byref(st)), "ghb_graph_bfs")
        if trace is not None:
            import numpy as np
            rows = min(trace_cap, st.levels)
            return depth, st.as_dict(), np.frombuffer(trace, dtype=np.float32).reshape(trace_cap, TRACE_COLS)[:rows].copy()
        return depth, st.as_dict()

    def bfs_many_host(self, srcs, out=None, max_depth=INT32_MAX, policy=POLICY_HEURISTIC, host_threads=0,
                      ws=None):
        """Depths from every source into a host array (numpy int32, n_src x
        n), the sources pipelined through the GPU, the copy engine and host
        threads.  Returns (array, stats); stats["device_ms"] is the call's
        wall time."""
        import numpy as np
        sh = np.ascontiguousarray(np.asarray(srcs, dtype=np.int32))
        if out is None:
            out = np.empty((len(sh), self.n), dtype=np.int32)
        if out.dtype != np.int32 or not out.flags.c_contiguous or out.size < len(sh) * self.n:
            raise ValueError("out must be a C-contiguous int32 array of n_src x n entries")
        opt = BfsOptions(policy=policy)
        st = TraversalStats()
        _check(lib().ghb_graph_bfs_many_host(_ws(ws), self._h, sh.ctypes.data_as(_p), len(sh), max_depth,
                                             out.ctypes.data_as(_p), host_threads, ctypes.byref(opt),
                                             ctypes.byref(st)), "ghb_graph_bfs_many_host")
        return out, st.as_dict()

    def bfs_pred(self, src, max_depth=INT32_MAX, ws=None):
        depth, pred = self._i32(), self._i32()
        st = TraversalStats()
        _check(lib().ghb_graph_bfs_pred(_ws(ws), self._h, src, max_depth, _ptr(depth), _ptr(pred), None,
                                        ctypes.byref(st)), "ghb_graph_bfs_pred")
        return depth, pred

    def msbfs(self, srcs, out=None, ws=None):
        sd = torch.as_tensor(srcs, dtype=torch.int32, device=self._dev)
        depth = out if out is not None else self._i32(len(sd))
        st = TraversalStats()
        _check(lib().ghb_graph_msbfs(_ws(ws), self._h, _ptr(sd), len(sd), _ptr(depth), ctypes.byref(st)),
               "ghb_graph_msbfs")
        return depth[: len(sd) * self.n].view(len(sd), self.n), st.as_dict()

    def msbfs_ex(self, srcs, schedule=None, trace_cap=0, out=None, ws=None):
        """Multi-source BFS with forced per-level directions (schedule: 0
        push, 1 pull per level; None: the rule) and a per-level trace of the
        first pass (rows: direction, ms, frontier vertices and out-entries,
        vertices and out-entries found).  Returns (depth, stats, trace)."""
        import numpy as np
        sd = torch.as_tensor(srcs, dtype=torch.int32, device=self._dev)
        depth = out if out is not None else self._i32(len(sd))
        opt = MsbfsOptions()
        sched = None
        if schedule is not None:
            sched = torch.as_tensor(list(schedule), dtype=torch.int8, device=self._dev)
            opt.schedule, opt.schedule_len = _ptr(sched), sched.numel()
        tr = None
        if trace_cap > 0:
            tr = torch.zeros(trace_cap * MS_TRACE_COLS, dtype=torch.float32, device=self._dev)
            opt.trace, opt.trace_cap = _ptr(tr), trace_cap
        st = TraversalStats()
        _check(lib().ghb_graph_msbfs_ex(_ws(ws), self._h, _ptr(sd), len(sd), _ptr(depth), ctypes.byref(opt),
                                        ctypes.byref(st)), "ghb_graph_msbfs_ex")
        trace = None
        if tr is not None:
            rows = min(trace_cap, st.levels)
            trace = tr.view(trace_cap, MS_TRACE_COLS)[:rows].cpu().numpy()
        return depth[: len(sd) * self.n].view(len(sd), self.n), st.as_dict(), trace

    def msbfs_reserve(self, n_src, ws=None):
        """Size the workspace for msbfs_launch with up to n_src sources."""
        _check(lib().ghb_graph_msbfs_reserve(_ws(ws), self._h, int(n_src)), "ghb_graph_msbfs_reserve")

    def msbfs_launch(self, srcs_dev, out, ws=None):
        """Launch-only multi-source BFS (one cooperative launch per 256
        sources; recordable in a CUDA graph): srcs_dev is an int32 device
        tensor, out an int32 device tensor of len(srcs_dev) * n entries."""
        _check(lib().ghb_graph_msbfs_launch(_ws(ws), self._h, _ptr(srcs_dev), srcs_dev.numel(), _ptr(out)),
               "ghb_graph_msbfs_launch")

    def mssssp(self, srcs, inf=DBL_MAX, out=None, ws=None):
        """Distances from every source (n_src x n), passes of up to 256."""
        sd = torch.as_tensor(srcs, dtype=torch.int32, device=self._dev)
        dist = out if out is not None else torch.empty(len(sd) * self.n, dtype=torch.float64, device=self._dev)
        st = TraversalStats()
        _check(lib().ghb_graph_mssssp(_ws(ws), self._h, _ptr(sd), len(sd), inf, _ptr(dist), ctypes.byref(st)),
               "ghb_graph_mssssp")
        return dist[: len(sd) * self.n].view(len(sd), self.n), st.as_dict()

    def sssp(self, src, inf=DBL_MAX, delta=0.0, policy=POLICY_HEURISTIC, trace=False, out=None, ws=None):
        """Distances and stats; with trace=True also the width-choice row
        (features, width used, rule's width, chosen by the network)."""
        dist = out if out is not None else torch.empty(self.n, dtype=torch.float64, device=self._dev)
        opt = SsspOptions(delta=delta, policy=policy)
        row = None
        if trace:
            row = (ctypes.c_float * TRACE_COLS)()
            opt.record_trace, opt.trace, opt.trace_cap = 1, ctypes.cast(row, _p), 1
        st = TraversalStats()
        _check(lib().ghb_graph_sssp(_ws(ws), self._h, src, inf, _ptr(dist), ctypes.byref(opt), ctypes.byref(st)),
               "ghb_graph_sssp")
        if row is not None:
            import numpy as np
            return dist, st.as_dict(), np.frombuffer(row, dtype=np.float32).copy()
        return dist, st.as_dict()

    def sssp_pred(self, src, inf=DBL_MAX, ws=None):
        dist = torch.empty(self.n, dtype=torch.float64, device=self._dev)
        pred = self._i32()
        st = TraversalStats()
        _check(lib().ghb_graph_sssp_pred(_ws(ws), self._h, src, inf, _ptr(dist), _ptr(pred), None,
                                         ctypes.byref(st)), "ghb_graph_sssp_pred")
        return dist, pred

    def wcc(self, out=None, ws=None):
        lab = out if out is not None else self._i32()
        _check(lib().ghb_graph_wcc(_ws(ws), self._h, _ptr(lab)), "ghb_graph_wcc")
        return lab

    def pagerank(self, iterations=10, damping=0.85, precision=PR_FP64, tolerance=0.0, l1_history=False, out=None,
                 ws=None):
        rank = out if out is not None else torch.empty(self.n, dtype=torch.float64, device=self._dev)
        hist = (ctypes.c_double * max(1, iterations))() if l1_history else None
        opt = PrOptions(iterations=iterations, damping=damping, precision=precision, tolerance=tolerance,
                        l1_history=ctypes.cast(hist, _p) if hist is not None else None)
        ran = _i32()
        _check(lib().ghb_graph_pagerank(_ws(ws), self._h, ctypes.byref(opt), _ptr(rank), ctypes.byref(ran)),
               "ghb_graph_pagerank")
        return rank, ran.value, (list(hist)[: ran.value] if hist is not None else None)

    def cdlp(self, iterations=10, out=None, ws=None):
        lab = out if out is not None else self._i32()
        _check(lib().ghb_graph_cdlp(_ws(ws), self._h, iterations, _ptr(lab)), "ghb_graph_cdlp")
        return lab

    def tc(self, ws=None):
        c64 = torch.empty(self.n, dtype=torch.int64, device=self._dev)
        c32 = self._i32()
        total = _i64()
        _check(lib().ghb_graph_tc(_ws(ws), self._h, _ptr(c64), _ptr(c32), ctypes.byref(total)), "ghb_graph_tc")
        return c64, c32, total.value


# ------------------------------------------------------------ schedule policy
def mlp_forward(params: torch.Tensor, norm: torch.Tensor, x: torch.Tensor, ws=None) -> torch.Tensor:
    """logits[B][20] of the policy network (device tensors, float32)."""
    logits = torch.empty(x.shape[0], POLICY_OUT, dtype=torch.float32, device=x.device)
    _check(lib().ghb_mlp_forward(_ws(ws), _ptr(params), _ptr(norm), _ptr(x.contiguous()), x.shape[0], _ptr(logits)),
           "ghb_mlp_forward")
    return logits


def mlp_grad(params: torch.Tensor, norm: torch.Tensor, x: torch.Tensor, y: torch.Tensor, weight=None, ws=None):
    """(gradient[6292], loss) of the summed per-head weighted mean cross-entropy."""
    grad = torch.empty(POLICY_PARAMS, dtype=torch.float32, device=x.device)
    loss = ctypes.c_float()
    _check(lib().ghb_mlp_grad(_ws(ws), _ptr(params), _ptr(norm), _ptr(x.contiguous()), _ptr(y.contiguous()),
                              _ptr(weight.contiguous()) if weight is not None else None, x.shape[0], _ptr(grad),
                              ctypes.byref(loss)), "ghb_mlp_grad")
    return grad, loss.value


def mlp_train(params: torch.Tensor, norm: torch.Tensor, x: torch.Tensor, y: torch.Tensor, epochs: int,
              lr: float = 3e-3, weight=None, ws=None):
    """Full-batch Adam on the device; updates params in place, returns the loss per epoch."""
    hist = (ctypes.c_float * max(1, epochs))()
    _check(lib().ghb_mlp_train(_ws(ws), _ptr(params), _ptr(norm), _ptr(x.contiguous()), _ptr(y.contiguous()),
                               _ptr(weight.contiguous()) if weight is not None else None, x.shape[0], epochs, lr,
                               ctypes.cast(hist, _p)), "ghb_mlp_train")
    return list(hist)[:epochs]


def policy_load(params, norm) -> None:
    """Install a network for POLICY_LEARNED (host or device float32 arrays);
    policy_load(None, None) uninstalls it."""
    if params is None and norm is None:
        _check(lib().ghb_policy_load(None, None), "ghb_policy_load")
        return
    p = torch.as_tensor(params, dtype=torch.float32).cpu().contiguous()
    q = torch.as_tensor(norm, dtype=torch.float32).cpu().contiguous()
    if p.numel() != POLICY_PARAMS or q.numel() != 2 * TRACE_FEATURES:
        raise ValueError("policy needs %d parameters and %d norm values" % (POLICY_PARAMS, 2 * TRACE_FEATURES))
    _check(lib().ghb_policy_load(ctypes.c_void_p(p.data_ptr()), ctypes.c_void_p(q.data_ptr())), "ghb_policy_load")


def policy_loaded() -> bool:
    return bool(lib().ghb_policy_loaded())


from .gpma import DynamicGraph, edge_keys  # noqa: E402
