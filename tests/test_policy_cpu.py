"""Host logic of the learned schedule policy: the per-level oracle (dynamic
program over the frontier's form) against brute force, the training rows,
and the training family."""
import itertools
import math

import numpy as np

from graphhet_b200 import policy as P


def brute_force(tq, tb, tc, tp):
    best = (math.inf, None)
    L = len(tq)
    for acts in itertools.product([P.PUSH_QUEUE, P.PUSH_BITMAP, P.PULL], repeat=L):
        if acts[0] == P.PULL:
            continue
        s, tot = 0, 0.0
        for l, a in enumerate(acts):
            comp = tc[l] if s == 1 else 0.0
            if a == P.PULL:
                tot += tp[l]
                s = 1
            else:
                tot += comp + (tq[l] if a == P.PUSH_QUEUE else tb[l])
                s = 0 if a == P.PUSH_QUEUE else 1
        if tot < best[0]:
            best = (tot, list(acts))
    return best


def test_oracle_schedule_matches_brute_force():
    rng = np.random.default_rng(1)
    for _ in range(200):
        L = int(rng.integers(1, 7))
        tq, tb, tc, tp = (rng.uniform(0.01, 1.0, L) for _ in range(4))
        if rng.random() < 0.3:
            tp[int(rng.integers(0, L))] = np.inf
        sched, cost, total = P.oracle_schedule(tq, tb, tc, tp)
        bt, bs = brute_force(tq, tb, tc, tp)
        assert math.isclose(total, bt, rel_tol=1e-12)
        assert math.isclose(sum(cost), total, rel_tol=1e-12)
        assert sched[0] != P.PULL


def test_level_rows_history_features_and_labels():
    L = 5
    trace = np.arange(L * 24, dtype=np.float32).reshape(L, 24)
    sched = [P.PUSH_QUEUE, P.PULL, P.PUSH_BITMAP, P.PUSH_QUEUE, P.PULL]
    cost = [0.1, 0.2, 0.3, 0.4, 0.5]
    X, Y = P.level_rows(trace, sched, cost)
    assert X.shape == (4, 12) and Y.shape == (4, 3)
    assert Y.tolist() == [[1, -1, -1], [0, 1, -1], [0, 0, -1], [1, -1, -1]]
    assert X[:, 9].tolist() == [0.0, 1.0, 0.0, 0.0]
    assert np.array_equal(X[:, :9], trace[1:, :9])
    assert np.array_equal(X[:, 10:], trace[1:, 10:12])


def test_level_rows_subsamples_long_traversals():
    L = 3000
    trace = np.zeros((L, 24), np.float32)
    trace[:, 3] = np.arange(L)
    sched = [P.PUSH_QUEUE] * L
    X, Y = P.level_rows(trace, sched, [0.01] * L, max_rows=48)
    assert len(X) <= 48
    assert X[:24, 3].tolist() == list(range(1, 25))
    assert X[-1, 3] == L - 1


def test_training_family():
    specs = P.training_specs(400)
    assert len(specs) == 400
    kinds = {k: [s for s in specs if s.kind == k] for k in ("rmat", "er", "grid", "powerlaw")}
    assert all(len(v) == 100 for v in kinds.values())
    assert all(16 <= s.scale <= 22 for s in specs)
    assert all(0.45 <= s.param <= 0.65 for s in kinds["rmat"])
    assert all(2.1 <= s.param <= 2.8 for s in kinds["powerlaw"])
    assert P.training_specs(400) == specs  # seeded


def test_init_params_layout():
    p = P.init_params(0)
    assert p.shape == (6292,) and p.dtype == np.float32
    assert np.all(p[768:832] == 0) and np.all(p[6272:] == 0)
    n = P.norm_of(np.random.default_rng(0).normal(size=(50, 12)).astype(np.float32))
    assert n.shape == (24,)


def test_level_weights_follow_the_cost_gap():
    r = dict(t_queue=np.array([1.0, 1.0, 1.0]), t_bitmap=np.array([1.0, 1.0, 1.0]),
             t_comp=np.array([0.0, 0.1, 0.1]), t_pull=np.array([np.inf, 5.0, 1.05]))
    sched, cost, total = P.oracle_schedule(r["t_queue"], r["t_bitmap"], r["t_comp"], r["t_pull"])
    w = P.level_weights(r, sched, total)
    assert w.shape == (3,) and np.all(w >= 0)
    assert w[1] > w[2]  # a wrong direction at level 1 costs 4 ms, at level 2 0.05 ms
    X, Y, W = P.level_rows(np.zeros((3, 24), np.float32), sched, cost, weights=w)
    assert len(W) == 2 and W[0] == np.float32(w[1])


def test_width_head_refit_keeps_bfs_decisions_and_learns_labels():
    """Refitting the SSSP width head touches only its 16 logits' weights:
    the shared layers and the BFS heads keep their values bit for bit, and
    the refit head follows labels that depend on the hidden features."""
    rng = np.random.default_rng(3)
    params = P.init_params(1)
    X = rng.normal(size=(300, 12)).astype(np.float32)
    norm = P.norm_of(X)
    H = P.hidden(params, norm, X)
    L = (H[:, :16].argmax(1)).astype(np.int32)  # a labelling the hidden layer can express
    out = P.refit_width_head(params, norm, X, L, np.ones(len(L), np.float32), epochs=1500)
    o3 = 12 * 64 + 64 + 64 * 64 + 64
    assert np.array_equal(out[:o3], params[:o3])
    W3o, W3p = out[o3:o3 + 1280].reshape(64, 20), params[o3:o3 + 1280].reshape(64, 20)
    assert np.array_equal(W3o[:, :4], W3p[:, :4])
    assert np.array_equal(out[o3 + 1280:o3 + 1284], params[o3 + 1280:o3 + 1284])
    assert P.width_accuracy(out, norm, X, L) > P.width_accuracy(params, norm, X, L) + 0.3


def test_ms_rows_features_labels_and_weights():
    """Rows of the multi-source direction model from one pass's traces:
    row r decides level r + 1 from the frontier trace row r expands, the
    frontier before it and the frontiers visited so far; the label is the
    faster direction, the weight what the other one costs."""
    n, m, k = 1024, 16384, 64
    tr = np.array([[0, 0.1, 1, 16, 40, 700],
                   [0, 0.2, 40, 700, 600, 9000],
                   [1, 0.3, 600, 9000, 100, 1500]], np.float32)
    t_push = np.array([0.10, 0.50, 0.20])
    t_pull = np.array([0.30, 0.20, 0.25])
    X, y, w = P.ms_rows(t_push, t_pull, tr, n, m, k, [0, 0, 1])
    assert X.shape == (3, P.MS_FEATURES)
    assert y.tolist() == [0.0, 1.0, 0.0]
    assert np.allclose(w, [0.20, 0.30, 0.05])
    # Row 1: frontier 40 vertices / 700 entries, after 1, visits 41, level 2.
    ref = P.ms_features(700, 40, 1, 41, n, m, k, 2, 0)
    assert np.allclose(X[1], ref)
    assert ref[4] == 0.25 and ref[6] == 0.0
    assert np.isclose(ref[0], np.log2(700 / m + 2.0**-30)) and np.isclose(ref[7], np.log2(41 / 2))


def test_ms_fit_learns_a_separable_direction():
    rng = np.random.default_rng(5)
    X = rng.normal(size=(500, P.MS_FEATURES))
    y = (X[:, 0] - 0.5 * X[:, 5] > 0.2).astype(np.float64)
    w = rng.uniform(0.1, 1.0, 500)
    th = P.fit_ms(X, y, w, epochs=4000)
    assert th.shape == (P.MS_FEATURES + 1,) and th.dtype == np.float32
    pred = (np.hstack([np.ones((500, 1)), X]) @ th) > 0
    assert (pred == (y > 0.5)).mean() > 0.95


def test_shipped_ms_model_has_nine_finite_weights():
    z = np.load(P.MS_WEIGHTS_PATH)
    wts = z["weights"]
    assert wts.shape == (P.MS_FEATURES + 1,) and np.all(np.isfinite(wts))
