"""The device edge-batch partition (dc_graph_kmax_edge_batches) numbers
every edge exactly as the host closed form and the oracle's restatement of
the reference's greedy loop (getKmaxEdgeBatches with KEDGE_BATCHING,
main.cu:1441-1488), on the graph's own kmax values."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _device_partition(g, frm, to):
    import torch
    dev = torch.device("cuda", 0)
    tf = torch.from_numpy(np.ascontiguousarray(frm, np.uint32).view(np.int32)).to(dev)
    tt = torch.from_numpy(np.ascontiguousarray(to, np.uint32).view(np.int32)).to(dev)
    out = torch.full((max(len(frm), 1),), -1, dtype=torch.int64, device=dev)
    torch.cuda.synchronize()
    n = g.kmax_edge_batches_device(tf.data_ptr(), tt.data_ptr(), len(frm), out.data_ptr())
    return n, out[:len(frm)].cpu().numpy()


@pytest.mark.parametrize("B,hot", [(1, False), (37, False), (5000, True), (5000, False), (300_000, True)])
def test_device_partition_matches_host_and_oracle(dc, orc, gpu, B, hot):
    V, s, d = dc.gen_rmat(14, 16, 4)
    rng = np.random.default_rng(B)
    with dc.Graph.from_edges(V, s, d) as g:
        g.decompose()
        kmaxes = g.kmaxes()
        frm = rng.integers(0, V, B).astype(np.uint32)
        to = rng.integers(0, V, B).astype(np.uint32)
        if hot:  # many edges into the few highest-kmax vertices: long runs of one root
            top = np.argsort(-kmaxes)[:8].astype(np.uint32)
            sel = rng.uniform(size=B) < 0.5
            to[sel] = top[rng.integers(0, 8, int(sel.sum()))]
        n_dev, got = _device_partition(g, frm, to)
        n_host, want = dc.kmax_edge_batches(kmaxes, frm, to)
        assert n_dev == n_host
        assert np.array_equal(got, want)
        if B <= 5000:
            n_or, want_or = orc.kedge_batches(V, kmaxes, frm, to)
            assert n_dev == n_or and np.array_equal(got, want_or)


def test_device_partition_after_maintenance_and_bad_ids(dc, gpu):
    V, s, d = dc.gen_rmat(12, 8, 2)
    with dc.Graph.from_edges(V, s, d) as g:
        g.decompose()
        u, v, dl = dc.gen_updates(V, s, d, 200, 0.7, 3)
        g.maintain(u, v, dl)
        kmaxes = g.kmaxes()
        ins = dl == 0
        n_dev, got = _device_partition(g, u[ins], v[ins])
        n_host, want = dc.kmax_edge_batches(kmaxes, u[ins], v[ins])
        assert n_dev == n_host and np.array_equal(got, want)
        with pytest.raises(dc.DCoreError) as e:
            _device_partition(g, np.array([0, V], np.uint32), np.array([1, 2], np.uint32))
        assert e.value.code == -1
        assert _device_partition(g, np.zeros(0, np.uint32), np.zeros(0, np.uint32))[0] == 0
