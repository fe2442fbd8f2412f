"""Edge cases of the newer entry points: empty and tiny graphs through row
ranges, row weights, the autotuner and the in-place row repair; a deletion
batch that empties the graph."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_empty_graph_ranges_and_tuning(dc, gpu):
    e = np.zeros(0, np.uint32)
    with dc.Graph.from_edges(5, e, e) as g:
        assert g.decompose_rows(0, 10) == (0, 0)
        assert list(g.row_weights()) == [0]
        assert np.array_equal(g.rows(0, 1), np.zeros((1, 5), np.int32))
        best, ms = g.autotune()
        assert g.tuning() == best
        assert not any(best["rows_split_permille"])  # kmax 0: nothing to split
        assert g.decompose() == (0, 0)


def test_tiny_cycle(dc, orc, gpu):
    # directed 3-cycle: every vertex has in- and out-degree 1
    s = np.array([0, 1, 2], np.uint32)
    d = np.array([1, 2, 0], np.uint32)
    okm, olm, okmaxes, orows = orc.dcore(3, s, d)
    with dc.Graph.from_edges(3, s, d) as g:
        assert g.decompose_rows(1, 1) == (okm, olm)
        assert np.array_equal(g.rows(1, 1), orows[1:2])
        best, _ = g.autotune()
        assert not any(best["rows_split_permille"])  # runs under 32 rows are never split
        assert g.decompose() == (okm, olm)
        assert np.array_equal(g.rows(), orows)


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_delete_every_edge(dc, orc, gpu, mode):
    V, s, d = dc.gen_rmat(9, 4, 3)
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_row_repair(mode)
        g.decompose()
        # in slices, the last one leaving an empty graph
        for a in range(0, len(s), 257):
            g.maintain(s[a:a + 257], d[a:a + 257], np.ones(len(s[a:a + 257]), np.uint8))
        assert g.info()[1] == 0
        assert g.decomp_info()["kmax"] == 0 and g.decomp_info()["lmax"] == 0
        assert not g.kmaxes().any()
        assert not g.rows().any()


def test_row_repair_mode_validation(dc, gpu):
    V, s, d = dc.gen_rmat(8, 4, 1)
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_row_repair(3)  # modes 0..3
        with pytest.raises(dc.DCoreError):
            g.set_row_repair(4)
        with pytest.raises(dc.DCoreError):
            g.set_row_repair(-1)


def test_reserve_device_memory(dc, gpu):
    dc.reserve_device_memory(0, 1 << 30)  # grows the pool; the memory stays for reuse
    with pytest.raises(dc.DCoreError):
        dc.reserve_device_memory(dc.device_count(), 1 << 20)
    V, s, d = dc.gen_rmat(10, 8, 3)
    with dc.Graph.from_edges(V, s, d) as g:  # allocations after the reservation work as before
        g.decompose()
