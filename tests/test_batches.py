"""Insert-batch partition (getKmaxEdgeBatches, KEDGE_BATCHING) against the
oracle's restatement of the reference's greedy loop."""
import numpy as np
import pytest


@pytest.mark.parametrize("seed", range(6))
def test_partition_matches_greedy_restatement(dc, orc, seed):
    rng = np.random.default_rng(seed)
    V = int(rng.integers(5, 200))
    kmaxes = rng.integers(0, 6, V).astype(np.int32)
    B = int(rng.integers(1, 400))
    frm = rng.integers(0, V, B).astype(np.uint32)
    to = rng.integers(0, V, B).astype(np.uint32)
    nb, got = dc.kmax_edge_batches(kmaxes, frm, to)
    onb, want = orc.kedge_batches(V, kmaxes, frm, to)
    assert nb == onb
    assert np.array_equal(got, want)


def test_partition_properties(dc):
    rng = np.random.default_rng(42)
    V = 1000
    kmaxes = rng.integers(0, 20, V).astype(np.int32)
    frm = rng.integers(0, V, 5000).astype(np.uint32)
    to = rng.integers(0, V, 5000).astype(np.uint32)
    nb, b = dc.kmax_edge_batches(kmaxes, frm, to)
    root = np.where(kmaxes[frm] > kmaxes[to], frm, to)
    for i in range(nb):
        sel = b == i
        assert sel.any()
        assert len(np.unique(kmaxes[root[sel]])) == 1          # one root kmax per sub-batch
        assert len(np.unique(root[sel])) == int(sel.sum())     # distinct roots
    # buckets appear in ascending root kmax
    first_k = [int(kmaxes[root[b == i]][0]) for i in range(nb)]
    assert first_k == sorted(first_k)


def test_partition_empty(dc):
    nb, b = dc.kmax_edge_batches(np.zeros(3, np.int32), np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert nb == 0 and len(b) == 0
