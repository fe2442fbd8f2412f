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


def _run_stream(dc, g, u, v, dl, sizes):
    pos, total = 0, 0.0
    for bs in sizes:
        st = g.maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], 0)
        total += st["total_ms"]
        pos += bs
    return total, pos


def test_trained_scheduler_gain_and_exactness(dc, orc, gpu):
    V, s, d = dc.gen_rmat(14, 16, 31)
    rng = np.random.default_rng(4)
    # training: the same stream on two handles, one per method
    tr_sizes = [int(x) for x in np.exp(rng.uniform(0, np.log(3000), 40))]
    u, v, dl = dc.gen_updates(V, s, d, sum(tr_sizes), 0.5, 41)
    logs = []
    for method in (1, 2):
        with dc.Graph.from_edges(V, s, d) as g:
            g.decompose()
            g.maint_log(True)
            pos = 0
            for bs in tr_sizes:
                g.maintain(u[pos:pos + bs], v[pos:pos + bs], dl[pos:pos + bs], method)
                pos += bs
            logs.append(g.maint_log())
    (fa, ma, ta), (fb, mb, tb) = logs
    assert np.allclose(fa, fb) and (ma == 1).all() and (mb == 2).all()
    X = fa
    # the methods differ in everything but the row recompute: learn that part
    T = np.log(np.stack([ta[:, 0] - ta[:, 2], tb[:, 0] - tb[:, 2]], 1).clip(1e-3) + 1e-2).astype(np.float32)
    mean, scale = X.mean(0), 1.0 / (X.std(0) + 1e-3)
    sched = dc.Scheduler(seed=11)
    sched.set_norm(mean, scale)
    loss = sched.train(X, T, np.ones_like(T, np.uint8), epochs=600, lr=3e-3)
    assert np.isfinite(loss)
    # evaluation on a fresh stream: learned policy vs the rule of thumb
    ev_sizes = [int(x) for x in np.exp(rng.uniform(0, np.log(3000), 25))]
    u2, v2, dl2 = dc.gen_updates(V, s, d, sum(ev_sizes), 0.5, 97)
    totals = {}
    finals = {}
    for name, sch in (("learned", sched), ("rule", None)):
        with dc.Graph.from_edges(V, s, d) as g:
            g.decompose()
            g.set_scheduler(sch)
            _run_stream(dc, g, u2, v2, dl2, ev_sizes)  # warm-up pass over a copy is not possible; time a second graph
        with dc.Graph.from_edges(V, s, d) as g:
            g.decompose()
            g.set_scheduler(sch)
            totals[name], n = _run_stream(dc, g, u2, v2, dl2, ev_sizes)
            finals[name] = (g.kmaxes(), g.rows())
    # exact either way: both equal a recomputation of the final graph
    cnt = Counter(zip(s.tolist(), d.tolist()))
    for a, b, x in zip(u2[:n].tolist(), v2[:n].tolist(), dl2[:n].tolist()):
        cnt[(a, b)] += -1 if x else 1
    es = [(a, b) for (a, b), m in cnt.items() for _ in range(m)]
    okm, olm, okmaxes, orows = orc.dcore(V, np.array([a for a, _ in es], np.uint32),
                                         np.array([b for _, b in es], np.uint32))
    for name in finals:
        assert np.array_equal(finals[name][0], okmaxes)
        assert np.array_equal(finals[name][1], orows)
    gain = totals["rule"] / totals["learned"]
    print(f"scheduler gain over the rule of thumb: {gain:.2f}x "
          f"(learned {totals['learned']:.1f} ms, rule {totals['rule']:.1f} ms)")
    assert gain > 0.8  # never much worse; the benchmark reports the measured gain
