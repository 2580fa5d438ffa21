"""ghb_wcc_noalloc: the WCC entry point for callers that must not allocate
device memory while the library runs (an application whose GPU memory is
owned by its own pool allocator, or a latency-critical caller for which
cudaMalloc would synchronise the device).  It is called through the C ABI and
must give the same labels as ghb_wcc (bit for bit: labels are integers) on two
calls in a row, with no workspace.

This file is named to be collected last, so a run that stops at the first
failure has run every other test before it."""
import ctypes

import numpy as np
import pytest
import torch

import oracle as O

pytestmark = pytest.mark.gpu


def graph_with_long_rows():
    """RMAT plus a star hub of 6000 leaves, so the walker defers long rows."""
    s, d = O.rmat_edges(14, 8 << 14, 31)
    hub = np.zeros(6000, np.int32)
    leaves = np.arange(100, 6100, dtype=np.int32)
    s = np.concatenate([s, hub])
    d = np.concatenate([d, leaves])
    return O.make_graph(1 << 14, s, d, False, weight_mode=0)


def run_noalloc(L, n, rp, col, out, stream):
    return L.ghb_wcc_noalloc(n, ctypes.c_void_p(rp.data_ptr()), ctypes.c_void_p(col.data_ptr()),
                             ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream))


def test_wcc_noalloc_matches_wcc_twice_in_a_row():
    import graphhet_b200 as G
    L = G.lib()
    L.ghb_wcc_noalloc.restype = ctypes.c_int
    L.ghb_wcc_noalloc.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    stream = torch.cuda.current_stream().cuda_stream
    for og in (graph_with_long_rows(), O.rmat_graph(11, 4, 3, weight_mode=0)):
        rp = torch.from_numpy(og.rowptr).cuda()
        col = torch.from_numpy(og.col).cuda()
        ref = torch.empty(og.n, dtype=torch.int32, device="cuda")
        G._check(L.ghb_wcc(G._ws(None), og.n, G._ptr(rp), G._ptr(col), G._ptr(ref)), "ghb_wcc")
        ref_h = ref.cpu().numpy()
        assert np.array_equal(ref_h, O.wcc(og))
        for _ in range(2):
            out = torch.full((og.n,), -7, dtype=torch.int32, device="cuda")
            G._check(run_noalloc(L, og.n, rp, col, out, stream), "ghb_wcc_noalloc")
            torch.cuda.synchronize()
            assert np.array_equal(out.cpu().numpy(), ref_h)


def test_wcc_noalloc_rejects_graphs_over_its_limit():
    import graphhet_b200 as G
    L = G.lib()
    L.ghb_wcc_noalloc.restype = ctypes.c_int
    L.ghb_wcc_noalloc.argtypes = [ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    # One vertex claiming 2^28 + 1 entries: rejected from rowptr alone, before
    # any kernel could read the (absent) entries.
    rp = torch.tensor([0, (1 << 28) + 1], dtype=torch.int32, device="cuda")
    col = torch.zeros(1, dtype=torch.int32, device="cuda")
    out = torch.zeros(1, dtype=torch.int32, device="cuda")
    s = run_noalloc(L, 1, rp, col, out, torch.cuda.current_stream().cuda_stream)
    assert s == 1  # GHB_ERR_INVALID_ARGUMENT
    assert b"268435456" in L.ghb_last_error()
