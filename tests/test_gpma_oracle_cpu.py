"""Pins the dynamic-graph oracle (oracle.gpma_update, the update semantics of
the reference's update_gpma, GPU_gpma.hpp:756-824): against one-at-a-time
application, against the reference's own graph_structure edits recorded in
tests/golden/gpma (make_golden.py), and, where the compiled reference is
present, against it live on fresh batches."""
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

FIX = os.path.join(GOLDEN, "gpma", "rmat9_seed42_batches.npz")


def dict_state(keys, vals):
    return dict(zip(keys.tolist(), vals.tolist()))


def random_batch(rng, n, keys, size):
    present = keys[rng.integers(len(keys), size=size // 3)] if len(keys) else np.zeros(0, np.int64)
    fresh = O.gpma_keys(rng.integers(n, size=size // 3), rng.integers(n, size=size // 3))
    bk = np.concatenate([present, fresh, present[: size // 6]])
    bv = np.where(rng.random(len(bk)) < 0.4, 0.0, rng.uniform(0.1, 3.0, len(bk)))
    perm = rng.permutation(len(bk))
    return bk[perm], bv[perm]


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_vectorised_matches_sequential(seed):
    rng = np.random.default_rng(seed)
    n = 300
    og = O.rmat_graph(8, 8, seed, directed=True)
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    state = dict_state(keys, vals)
    for _ in range(5):
        bk, bv = random_batch(rng, n, keys, 600)
        keys, vals, counts = O.gpma_update(keys, vals, bk, bv)
        state = O.gpma_update_sequential(state, bk, bv)
        assert dict_state(keys, vals) == state
        assert np.all(np.diff(keys) > 0)
        assert sum(counts) == len(bk)


def test_edge_cases():
    keys = O.gpma_keys([0, 0, 2], [1, 3, 0])
    vals = np.array([1.0, 2.0, 3.0])
    # empty batch
    k, v, c = O.gpma_update(keys, vals, np.zeros(0, np.int64), np.zeros(0))
    assert np.array_equal(k, keys) and np.array_equal(v, vals) and c == (0, 0, 0, 0)
    # delete absent, delete present, modify, insert, repeat (last wins: insert then delete -> nothing)
    bk = O.gpma_keys([1, 0, 2, 1, 3, 3], [1, 3, 0, 2, 3, 3])
    bv = np.array([0.0, 0.0, 7.0, 5.0, 4.0, 0.0])
    k, v, c = O.gpma_update(keys, vals, bk, bv)
    assert dict_state(k, v) == {int(O.gpma_keys([0], [1])[0]): 1.0, int(O.gpma_keys([2], [0])[0]): 7.0,
                                int(O.gpma_keys([1], [2])[0]): 5.0}
    assert c == (1, 1, 1, 3)
    # everything deleted
    k, v, c = O.gpma_update(keys, vals, keys, np.zeros(3))
    assert len(k) == 0 and c == (0, 3, 0, 0)


def test_oracle_matches_reference_fixture():
    z = np.load(FIX)
    n = int(z["n"])
    keys, vals = O.gpma_from_csr(z["rowptr"], z["col"], z["w"])
    for i in range(4):
        keys, vals, _ = O.gpma_update(keys, vals, O.gpma_keys(z[f"b{i}_src"], z[f"b{i}_dst"]), z[f"b{i}_w"])
        rp, col, w = O.gpma_to_csr(n, keys, vals)
        assert np.array_equal(rp, z[f"a{i}_rowptr"])
        assert np.array_equal(col, z[f"a{i}_col"])
        assert np.array_equal(w, z[f"a{i}_w"])


@pytest.mark.skipif(not O.ref_available(), reason="compiled reference (oracle/_ref) not built")
def test_oracle_matches_compiled_reference_live():
    import sys
    sys.path.insert(0, GOLDEN)
    import make_golden as M
    og = O.rmat_graph(10, 8, 77, directed=True)
    r = O.Ref().load(og)
    keys, vals = O.gpma_from_csr(og.rowptr, og.col, og.w)
    for s, d, w in M.gpma_batches(og.rowptr, og.col, og.n, 3, 3000, 5):
        r.apply_updates(s, d, w)
        keys, vals, _ = O.gpma_update(keys, vals, O.gpma_keys(s, d), w)
        rp, col, ww = r.export_out()
        ork, orv = O.gpma_from_csr(rp, col, ww)
        assert np.array_equal(ork, keys) and np.array_equal(orv, vals)
    r.close()


def test_planted_mistake_is_caught():
    """'First occurrence wins' instead of last: the fixture must reject it."""
    z = np.load(FIX)
    keys, vals = O.gpma_from_csr(z["rowptr"], z["col"], z["w"])
    bk = O.gpma_keys(z["b0_src"], z["b0_dst"])
    bv = z["b0_w"]
    # Reverse the batch: a repeated key now keeps its first value.
    k2, v2, _ = O.gpma_update(keys, vals, bk[::-1], bv[::-1])
    rp, col, w = O.gpma_to_csr(int(z["n"]), k2, v2)
    same = (np.array_equal(rp, z["a0_rowptr"]) and np.array_equal(col, z["a0_col"])
            and np.array_equal(w, z["a0_w"]))
    assert not same
