"""The C ABI library loads without a GPU and exports every entry point that
include/ghb.h declares (no compute calls here)."""
import ctypes
import os
import re

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "ghb.h")
LIB = os.path.join(ROOT, "graphhet_b200", "libghb.so")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = re.findall(r"\b(ghb_[a-z0-9_]+)\s*\(", text)
    return sorted(set(names))


def test_header_declares_the_reference_entry_points():
    names = declared_functions()
    for required in ["ghb_bfs", "ghb_bfs_pred", "ghb_sssp", "ghb_sssp_pred", "ghb_wcc", "ghb_pagerank",
                     "ghb_cdlp", "ghb_tc", "ghb_csr_build", "ghb_msbfs", "ghb_batch_wcc", "ghb_batch_tc"]:
        assert required in names


def test_library_exports_every_declared_symbol():
    assert os.path.exists(LIB), "build libghb.so first (make)"
    L = ctypes.CDLL(LIB)
    missing = [n for n in declared_functions() if not hasattr(L, n)]
    assert not missing, f"declared but not exported: {missing}"


def test_version_and_status_strings():
    L = ctypes.CDLL(LIB)
    L.ghb_status_string.restype = ctypes.c_char_p
    assert L.ghb_version() >= 10000
    assert L.ghb_status_string(0) == b"ok"
    assert L.ghb_status_string(4) == b"device wait timed out"


def test_python_layer_fails_loudly_without_library(monkeypatch, tmp_path):
    import graphhet_b200 as G
    monkeypatch.setattr(G, "LIB_PATH", str(tmp_path / "missing.so"))
    monkeypatch.setattr(G, "_lib", None)
    with pytest.raises(G.GhbError):
        G.lib()
