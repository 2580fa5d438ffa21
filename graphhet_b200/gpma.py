"""Dynamic graph: batched edge inserts, deletes and weight changes on a
GPU-resident graph (libghb's ghb_gpma_*), the counterpart of the reference's
GPMA (include/GPU_gpma/GPU_gpma.hpp).

Update semantics are update_gpma's (GPU_gpma.hpp:756-824): a key is
(row << 32) | col; value 0 deletes the entry when present; any other value
sets the weight of a present entry or inserts it.  Repeated keys in a batch:
the last one wins.  The analytics of this package run on the compact CSR of
`csr_graph()` (rows sorted, rebuilt after each change)."""
from __future__ import annotations

import ctypes
from typing import Dict, Optional, Tuple

import torch

from . import CSRGraph, GhbError, _check, _i32, _i64, _p, _ptr, _ws, lib

STAT_NAMES = ("batches", "inserted", "deleted", "modified", "rows_moved", "repacks", "slots_used", "slots")


def edge_keys(src: torch.Tensor, dst: torch.Tensor) -> torch.Tensor:
    """int64 keys (src << 32) | dst, the bit pattern of the reference's
    KEY_TYPE (LDBC_GPU_gpma.cu:91-93)."""
    return (src.to(torch.int64) << 32) | dst.to(torch.int64)


class DynamicGraph:
    """A GPU-resident graph over n vertices that takes batches of updates."""

    def __init__(self, n: int, ws=None):
        self._ws = ws
        self._h = _p()
        _check(lib().ghb_gpma_create(_ws(ws), int(n), ctypes.byref(self._h)), "ghb_gpma_create")

    @classmethod
    def from_csr(cls, rowptr: torch.Tensor, col: torch.Tensor, w: Optional[torch.Tensor] = None, ws=None):
        """Load a CSR (rows strictly increasing, weights nonzero; w None
        means weight 1), like init_gpma_from_csr (GPU_gpma.hpp:851-909)."""
        g = cls(int(rowptr.numel()) - 1, ws=ws)
        _check(lib().ghb_gpma_load_csr(_ws(ws), g._h, _ptr(rowptr), _ptr(col) if col.numel() else None,
                                       _ptr(w) if w is not None and w.numel() else None), "ghb_gpma_load_csr")
        return g

    @classmethod
    def from_graph(cls, g: CSRGraph, weights: bool = True, ws=None):
        return cls.from_csr(g.rowptr, g.col, g.w if weights else None, ws=ws)

    def close(self) -> None:
        if self._h:
            lib().ghb_gpma_destroy(self._h)
            self._h = _p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def clone(self) -> "DynamicGraph":
        out = DynamicGraph.__new__(DynamicGraph)
        out._ws = self._ws
        out._h = _p()
        _check(lib().ghb_gpma_clone(_ws(self._ws), self._h, ctypes.byref(out._h)), "ghb_gpma_clone")
        return out

    def clear(self) -> None:
        _check(lib().ghb_gpma_clear(_ws(self._ws), self._h), "ghb_gpma_clear")

    def update(self, keys: torch.Tensor, values: torch.Tensor) -> Dict[str, int]:
        """Apply one batch (device int64 keys, float64 values)."""
        if keys.numel() != values.numel():
            raise GhbError("keys and values differ in length")
        keys = keys.to(torch.int64).contiguous()
        values = values.to(torch.float64).contiguous()
        t = (_i64 * 4)()
        _check(lib().ghb_gpma_update(_ws(self._ws), self._h, _ptr(keys) if keys.numel() else None,
                                     _ptr(values) if values.numel() else None, int(keys.numel()), t),
               "ghb_gpma_update")
        return dict(zip(("inserted", "deleted", "modified", "ignored"), [int(x) for x in t]))

    def insert_edges(self, src: torch.Tensor, dst: torch.Tensor, w: Optional[torch.Tensor] = None):
        """batch_add_edge of the LDBC driver (LDBC_GPU_gpma.cu:142-144): weight 1 unless given."""
        v = torch.ones(src.numel(), dtype=torch.float64, device=src.device) if w is None else w
        return self.update(edge_keys(src, dst), v)

    def delete_edges(self, src: torch.Tensor, dst: torch.Tensor):
        """batch_delete_edge (LDBC_GPU_gpma.cu:146-148): value VALUE_NONE = 0."""
        return self.update(edge_keys(src, dst), torch.zeros(src.numel(), dtype=torch.float64, device=src.device))

    def find(self, keys: torch.Tensor) -> torch.Tensor:
        keys = keys.to(torch.int64).contiguous()
        out = torch.empty(max(1, keys.numel()), dtype=torch.float64, device=keys.device)
        _check(lib().ghb_gpma_find(_ws(self._ws), self._h, _ptr(keys) if keys.numel() else None,
                                   int(keys.numel()), _ptr(out)), "ghb_gpma_find")
        return out[: keys.numel()]

    def info(self) -> Tuple[int, int, int, int]:
        n, m, slots, ver = _i32(), _i64(), _i64(), _i64()
        _check(lib().ghb_gpma_info(self._h, ctypes.byref(n), ctypes.byref(m), ctypes.byref(slots),
                                   ctypes.byref(ver)), "ghb_gpma_info")
        return n.value, m.value, slots.value, ver.value

    @property
    def n(self) -> int:
        return self.info()[0]

    @property
    def m(self) -> int:
        return self.info()[1]

    def stats(self) -> Dict[str, int]:
        s = (_i64 * 8)()
        _check(lib().ghb_gpma_stats(self._h, s), "ghb_gpma_stats")
        return dict(zip(STAT_NAMES, [int(x) for x in s]))

    def csr_view(self, weights: bool = False):
        """(rowptr, col, w) device pointers of the cached snapshot, as ints."""
        rp, col, w = _p(), _p(), _p()
        _check(lib().ghb_gpma_csr(_ws(self._ws), self._h, int(weights), ctypes.byref(rp), ctypes.byref(col),
                                  ctypes.byref(w)), "ghb_gpma_csr")
        return rp.value, col.value, w.value

    def csr_graph(self, weights: bool = True, directed: bool = False, in_graph: Optional["DynamicGraph"] = None,
                  device=None) -> CSRGraph:
        """A copy of the current graph as a CSRGraph.  Undirected (the
        default): the rows hold both directions.  Directed: the in-rows come
        from `in_graph` (the reference keeps an in-GPMA beside the out-GPMA,
        LDBC_GPU_gpma.cu:155-211) or, without one, from a transpose."""
        n, m, _, _ = self.info()
        dev = device or torch.device("cuda", torch.cuda.current_device())
        rp = torch.empty(n + 1, dtype=torch.int32, device=dev)
        col = torch.empty(max(1, m), dtype=torch.int32, device=dev)
        w = torch.empty(max(1, m), dtype=torch.float64, device=dev) if weights else None
        _check(lib().ghb_gpma_export(_ws(self._ws), self._h, _ptr(rp), _ptr(col), _ptr(w)), "ghb_gpma_export")
        g = CSRGraph(n=n, rowptr=rp, col=col[:m], w=w[:m] if w is not None else None, directed=directed)
        if directed:
            if in_graph is not None:
                ig = in_graph.csr_graph(weights=weights, device=dev)
                if ig.n != n:
                    raise GhbError("in_graph has a different vertex count")
                g.in_rowptr, g.in_col, g.in_w = ig.rowptr, ig.col, ig.w
            else:
                from . import transpose_csr
                g.in_rowptr, g.in_col, g.in_w = transpose_csr(n, g.rowptr, g.col, g.w, ws=self._ws)
        return g
