"""Row sharding on one GPU: the ranges a multi-GPU run would give to its
ranks, computed one after another on one device (ranks never wait on one
another, so this is exactly their work), together equal the oracle's full
decomposition."""
import numpy as np
import pytest

import dcore_dist

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("scale,ef,seed,world", [(12, 8, 1, 2), (14, 16, 2, 4), (15, 16, 3, 8)])
def test_row_ranges_cover_full_decomposition(dc, orc, gpu, scale, ef, seed, world):
    V, s, d = dc.gen_rmat(scale, ef, seed)
    K, L, ref_km, ref_rows = orc.dcore(V, s, d)
    with dc.Graph.from_edges(V, s, d) as g:
        k, l = g.decompose_rows(1, 0)  # kmax and row 0 only
        assert (k, l) == (K, L)
        assert np.array_equal(g.kmaxes(), ref_km)
        w = g.row_weights()
        assert len(w) == K + 1 and (np.diff(w.astype(np.int64)) <= 0).all()
        assert int(w[0]) == 2 * len(s)
        shards = dcore_dist.row_shards(w, world)
        assert len(shards) == world
        covered = []
        for first, last in shards:
            if first > last:
                continue
            g.decompose_rows(first, last)
            got = g.rows(first, last - first + 1)
            assert np.array_equal(got, ref_rows[first:last + 1]), (first, last)
            assert np.array_equal(g.rows(0, 1)[0], ref_rows[0])
            covered += list(range(first, last + 1))
        assert covered == list(range(1, K + 1))


def test_rows_outside_the_range_are_refused(dc, gpu):
    V, s, d = dc.gen_rmat(12, 16, 5)
    with dc.Graph.from_edges(V, s, d) as g:
        K, _ = g.decompose_rows(0, 0)
        assert K >= 4
        g.decompose_rows(2, 3)
        g.rows(2, 2)
        with pytest.raises(dc.DCoreError):
            g.rows(1, 1)
        with pytest.raises(dc.DCoreError):
            g.rows(3, 2)
        with pytest.raises(dc.DCoreError):
            g.skyline()
        # maintenance needs every row: it decomposes fully first
        u, v, dl = dc.gen_updates(V, s, d, 10, 0.5, 1)
        g.maintain(u, v, dl)
        g.skyline()
