"""Learned maintenance scheduler: the BF16 MLP kernels against a float64
numpy reference (BF16 rounding of inputs, weights and activations
emulated), training, and what the trained network gains over the rule of
thumb on a fresh update stream.  Maintenance results stay exact either way."""
from collections import Counter

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def bf16(a):
    a = np.ascontiguousarray(a, np.float32)
    b = a.view(np.uint32).astype(np.uint64)
    b = ((b + 0x7FFF + ((b >> 16) & 1)) >> 16) << 16
    return b.astype(np.uint32).view(np.float32).astype(np.float64)


def unpack(p):
    o = 0
    def take(n, shape):
        nonlocal o
        x = p[o:o + n].reshape(shape)
        o += n
        return x
    W1 = take(64 * 16, (64, 16)); b1 = take(64, (64,))
    W2 = take(64 * 64, (64, 64)); b2 = take(64, (64,))
    W3 = take(2 * 64, (2, 64)); b3 = take(2, (2,))
    return W1, b1, W2, b2, W3, b3


def ref_forward(p, X):
    W1, b1, W2, b2, W3, b3 = [bf16(a) for a in unpack(p)]
    xb = bf16(X)
    a1 = xb @ W1.T + b1
    h1 = bf16(np.maximum(a1, 0))
    a2 = h1 @ W2.T + b2
    h2 = bf16(np.maximum(a2, 0))
    y = h2 @ W3.T + b3
    return xb, a1, h1, a2, h2, y


def ref_grad(p, X, T, M):
    W1, b1, W2, b2, W3, b3 = [bf16(a) for a in unpack(p)]
    xb, a1, h1, a2, h2, y = ref_forward(p, X)
    n_on = max(M.sum(), 1)
    dy = 2 * (y - T) * M / n_on
    loss = float(((y - T) ** 2 * M).sum() / n_on)
    gW3 = dy.T @ h2; gb3 = dy.sum(0)
    d2 = (dy @ W3) * (h2 > 0)
    gW2 = d2.T @ h1; gb2 = d2.sum(0)
    d1 = (d2 @ W2) * (h1 > 0)
    gW1 = d1.T @ xb; gb1 = d1.sum(0)
    return np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3.ravel(), gb3]), loss


def test_forward_matches_reference(dc, gpu):
    s = dc.Scheduler(seed=3)
    rng = np.random.default_rng(0)
    X = rng.normal(size=(300, 16)).astype(np.float32)
    Y = s.predict(X)
    want = ref_forward(s.params(), X)[-1]
    assert np.allclose(Y, want, rtol=2e-2, atol=2e-2), np.abs(Y - want).max()


def test_gradients_match_float64_reference(dc, gpu):
    s = dc.Scheduler(seed=5)
    rng = np.random.default_rng(1)
    X = rng.normal(size=(200, 16)).astype(np.float32)
    T = rng.normal(size=(200, 2)).astype(np.float32)
    M = (rng.random((200, 2)) < 0.8).astype(np.uint8)
    g, loss = s.grad(X, T, M)
    gref, lref = ref_grad(s.params(), X, T, M)
    assert abs(loss - lref) <= 1e-3 * max(1.0, abs(lref))
    rel = np.linalg.norm(g - gref) / np.linalg.norm(gref)
    assert rel < 2e-2, rel
    # per-layer check as well
    for a, b in zip(unpack(g), unpack(gref)):
        assert np.linalg.norm(a - b) <= 5e-2 * np.linalg.norm(b) + 1e-6


def test_training_fits_a_regression(dc, gpu):
    s = dc.Scheduler(seed=7)
    rng = np.random.default_rng(2)
    X = rng.normal(size=(512, 16)).astype(np.float32)
    T = np.stack([np.sin(X[:, 0]) + 0.5 * X[:, 1], X[:, 2] ** 2 - X[:, 3]], 1).astype(np.float32)
    M = np.ones((512, 2), np.uint8)
    _, l0 = s.grad(X, T, M)
    l1 = s.train(X, T, M, epochs=400, lr=3e-3)
    assert l1 < 0.2 * l0, (l0, l1)


def _hot_stream(dc, V, s, d, sizes, rng, seed, hot_frac=0.2):
    od = np.bincount(s, minlength=V)
    hot = np.argsort(-od, kind="stable")[:max(1, V // 100)].astype(np.uint32)
    hot_batch = rng.uniform(size=len(sizes)) < hot_frac
    op_hot = np.repeat(hot_batch.astype(np.uint8), sizes)
    return dc.gen_updates_hot(V, s, d, int(np.sum(sizes)), 0.5, seed, hot, op_hot)


PATHS = ((1, 3), (2, 0))  # (method, row mode): incremental (local, rows in place), full (re-peel, rows recomputed)


def _per_path_log(dc, V, s, d, u, v, dl, sizes, paths=PATHS):
    """The stream on one copy per path: features and device times (one log
    record per batch, split batches included)."""
    logs = []
    for method, mode in paths:
        with dc.Graph.from_edges(V, s, d, gap_min=2, gap_div=16) as g:
            g.set_row_repair(mode)
            g.decompose()
            g.maint_log(True)
            pos = 0
            for bs in sizes:
                g.maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], method)
                pos += bs
            logs.append(g.maint_log())
    feats = [f for f, _, _ in logs]
    for f in feats[1:]:
        assert np.allclose(f, feats[0])
    return feats[0], [t for _, _, t in logs]


def _rule_times(dc, V, s, d, u, v, dl, sizes):
    """The rule of thumb's own run (no network, the default row mode)."""
    ms = []
    with dc.Graph.from_edges(V, s, d, gap_min=2, gap_div=16) as g:
        g.decompose()
        pos = 0
        for bs in sizes:
            ms.append(g.maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], 0)["total_ms"])
            pos += bs
    return np.array(ms)


def test_trained_scheduler_gain_and_exactness(dc, orc, gpu):
    rng = np.random.default_rng(4)
    # training log over graphs of three sizes: each batch timed on the
    # incremental and on the full path
    Xs, Ts = [], []
    for j, scale in enumerate((12, 13, 14)):
        V, s, d = dc.gen_rmat(scale, 16, 31 + j)
        sizes = [int(x) for x in np.exp(rng.uniform(0, np.log(4000), 30))]
        u, v, dl = _hot_stream(dc, V, s, d, sizes, rng, 41 + j)
        X, (ta, tb) = _per_path_log(dc, V, s, d, u, v, dl, sizes)
        Xs.append(X)
        Ts.append(np.log(np.stack([ta[:, 0], tb[:, 0]], 1).clip(1e-3)))
    X = np.concatenate(Xs).astype(np.float32)
    T = np.concatenate(Ts).astype(np.float32)
    sched = dc.Scheduler(seed=11)
    sched.set_norm(X.mean(0), 1.0 / (X.std(0) + 1e-3))
    loss = sched.train(X, T, np.ones_like(T, np.uint8), epochs=800, lr=3e-3)
    assert np.isfinite(loss)
    # evaluation on a fresh graph and stream: both paths timed on every
    # batch (the network is charged the time of the path it picks; every
    # path leaves the same decomposition), the rule of thumb on its own run
    V, s, d = dc.gen_rmat(14, 16, 97)
    ev_sizes = [int(x) for x in np.exp(rng.uniform(0, np.log(4000), 30))]
    u2, v2, dl2 = _hot_stream(dc, V, s, d, ev_sizes, rng, 98)
    Xe, (ta, tb) = _per_path_log(dc, V, s, d, u2, v2, dl2, ev_sizes)
    t = np.stack([ta[:, 0], tb[:, 0]], 1)
    learned = np.argmin(sched.predict(Xe), 1)
    t_learned = t[np.arange(len(t)), learned].sum()
    t_rule = _rule_times(dc, V, s, d, u2, v2, dl2, ev_sizes).sum()
    t_best = t.min(1).sum()
    gain = t_rule / t_learned
    print(f"scheduler gain over the rule of thumb: {gain:.2f}x (learned {t_learned:.1f} ms, "
          f"rule {t_rule:.1f} ms, best of the two paths {t_best:.1f} ms)")
    # the network's picks cost within 15 % of the per-batch best of the two
    # paths (same timings: no run-to-run noise), and it loses nothing that
    # matters against the rule of thumb's own run (measured apart: 10 % slack
    # for timing noise between runs)
    assert t_learned <= 1.15 * t_best
    assert gain >= 0.9
    # exactness with the network attached: equal to a recomputation
    with dc.Graph.from_edges(V, s, d) as g:
        g.decompose()
        g.set_scheduler(sched)
        pos = 0
        for bs in ev_sizes:
            st = g.maintain(u2[pos:pos + bs], v2[pos:pos + bs], dl2[pos:pos + bs], 0)
            assert st["method"] in (1, 2)
            pos += bs
        km, rows = g.kmaxes(), g.rows()
    cnt = Counter(zip(s.tolist(), d.tolist()))
    for a, b, x in zip(u2[:pos].tolist(), v2[:pos].tolist(), dl2[:pos].tolist()):
        cnt[(a, b)] += -1 if x else 1
    es = [(a, b) for (a, b), m in cnt.items() for _ in range(m)]
    okm, olm, okmaxes, orows = orc.dcore(V, np.array([a for a, _ in es], np.uint32),
                                         np.array([b for _, b in es], np.uint32))
    assert np.array_equal(km, okmaxes)
    assert np.array_equal(rows, orows)
