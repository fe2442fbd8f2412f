"""Serving loop: many graphs, interleaved update requests, continuous
batching on several workers under an HBM budget small enough to force
evictions.  Every graph's decomposition after its requests must equal
(a) the same requests applied to that graph alone, one request per
maintenance call, and (b) the oracle on the final edge set."""
from collections import Counter

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _apply(cnt, u, v, dl):
    for a, b, x in zip(u.tolist(), v.tolist(), dl.tolist()):
        if x:
            cnt[(a, b)] -= 1
            if cnt[(a, b)] == 0:
                del cnt[(a, b)]
        else:
            cnt[(a, b)] += 1


def _edges(cnt):
    s, d = [], []
    for (a, b), m in cnt.items():
        s += [a] * m
        d += [b] * m
    return np.array(s, np.uint32), np.array(d, np.uint32)


def _workload(dc, n_graphs, seed):
    rng = np.random.default_rng(seed)
    graphs, streams = [], []
    for i in range(n_graphs):
        scale = int(rng.integers(9, 13))
        ef = int(rng.choice([8, 16, 32]))
        V, s, d = dc.gen_rmat(scale, ef, seed * 100 + i)
        n_ops = int(rng.integers(200, 600))
        u, v, dl = dc.gen_updates(V, s, d, n_ops, 0.6, seed * 100 + 50 + i)
        # split into requests of 1..64 updates (log-uniform sizes)
        cuts, pos = [], 0
        while pos < n_ops:
            k = int(np.exp(rng.uniform(0, np.log(64))))
            cuts.append((pos, min(n_ops, pos + k)))
            pos += k
        graphs.append((V, s, d))
        streams.append([(u[a:b], v[a:b], dl[a:b]) for a, b in cuts])
    # interleave requests of all graphs in a random arrival order
    order = [(g, j) for g in range(n_graphs) for j in range(len(streams[g]))]
    rng.shuffle(order)
    nxt = [0] * n_graphs
    arrival = []
    for g, _ in order:  # keep each graph's own requests in order
        arrival.append((g, nxt[g]))
        nxt[g] += 1
    return graphs, streams, arrival


@pytest.mark.parametrize("workers", [1, 4])
def test_mix_matches_alone_and_oracle(dc, orc, gpu, workers):
    graphs, streams, arrival = _workload(dc, 8, 7)
    # budget: room for about three of the graphs at once
    sizes = []
    for V, s, d in graphs:
        with dc.Graph.from_edges(V, s, d) as g:
            g.decompose()
            sizes.append(g.device_bytes())
    budget = int(sum(sorted(sizes)[-3:]) * 1.2)
    with dc.Server(budget, max_concurrent=workers) as srv:
        ids = [srv.add_graph(V, s, d) for V, s, d in graphs]
        for g, j in arrival:
            u, v, dl = streams[g][j]
            srv.submit(ids[g], u, v, dl)
        srv.drain()
        comp = srv.completions()
        info = srv.info()
        n_req = sum(len(x) for x in streams)
        assert len(comp["id"]) == n_req and info["completed"] == n_req
        assert (comp["status"] == 0).all()
        assert sorted(comp["id"].tolist()) == list(range(1, n_req + 1))
        assert info["evictions"] > 0, info
        assert info["peak_bytes"] <= budget, info
        results = [srv.result(ids[g], graphs[g][0]) for g in range(len(graphs))]
    for gi, (V, s, d) in enumerate(graphs):
        cnt = Counter(zip(s.tolist(), d.tolist()))
        with dc.Graph.from_edges(V, s, d) as g:
            g.decompose()
            for u, v, dl in streams[gi]:
                g.maintain(u, v, dl)
                _apply(cnt, u, v, dl)
            alone_k, alone_r = g.kmaxes(), g.rows()
        km, rows = results[gi]
        assert np.array_equal(km, alone_k), f"graph {gi}: kmax differs from the graph alone"
        assert np.array_equal(rows, alone_r), f"graph {gi}: rows differ from the graph alone"
        fs, fd = _edges(cnt)
        okm, olm, okmaxes, orows = orc.dcore(V, fs, fd)
        assert np.array_equal(km, okmaxes)
        assert np.array_equal(rows, orows)


def test_coalescing_and_latency(dc, gpu):
    # one graph, many requests queued before any worker can start: the
    # worker coalesces them; every request reports its batch
    V, s, d = dc.gen_rmat(12, 8, 3)
    u, v, dl = dc.gen_updates(V, s, d, 400, 0.6, 4)
    with dc.Server(8 << 30, max_concurrent=1) as srv:
        gid = srv.add_graph(V, s, d)
        for i in range(0, 400, 4):
            srv.submit(gid, u[i:i + 4], v[i:i + 4], dl[i:i + 4])
        srv.drain()
        c = srv.completions()
        assert len(c["id"]) == 100
        assert c["batch_requests"].max() > 1  # requests were coalesced
        assert (c["latency_ms"] > 0).all()
        # batch_updates is consistent with batch_requests of 4 updates each
        assert np.array_equal(c["batch_updates"], 4 * c["batch_requests"].astype(np.uint64))
        assert srv.info()["batches"] < 100


def test_bad_requests_rejected(dc, gpu):
    V, s, d = dc.gen_rmat(8, 4, 1)
    with dc.Server(1 << 30) as srv:
        gid = srv.add_graph(V, s, d)
        with pytest.raises(dc.DCoreError):
            srv.submit(gid + 1, np.array([0], np.uint32), np.array([1], np.uint32))
        with pytest.raises(dc.DCoreError):
            srv.submit(gid, np.array([V], np.uint32), np.array([1], np.uint32))
        srv.drain(1000)
