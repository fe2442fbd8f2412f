"""Launch shapes change speed, never answers: the decomposition under several
peel grids, chunk sizes, row-kernel grids and splits of the rows over two
concurrent launches equals the default one, maintenance stays exact with the
rows split, and the autotuner leaves a valid setting and a full
decomposition behind."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SETTINGS = [(1, 1, 16, []), (2, 1, 32, [300]), (1, 2, 128, [500]), (4, 4, 256, []), (3, 2, 4096, [900]),
            (2, 3, 64, [1]), (2, 2, 64, [200, 450]), (3, 3, 64, [150, 400, 700]), (1, 1, 32, [1, 2, 999]),
            (2, 2, 64, [100, 200, 300, 400, 500, 600, 700]), (1, 1, 64, [50, 100, 150, 200, 250, 300, 350])]


def test_settings_give_identical_results(dc, gpu):
    V, s, d = dc.gen_rmat(15, 16, 9)
    with dc.Graph.from_edges(V, s, d) as g:
        K, L = g.decompose()
        ref_km, ref_rows, ref_sky = g.kmaxes(), g.rows(), g.skyline()
        for pb, rb, ch, sp in SETTINGS:
            g.set_tuning(pb, rb, ch, sp)
            assert g.tuning() == {"peel_blocks_per_sm": pb, "rows_blocks_per_sm": rb, "peel_chunk": ch,
                                  "rows_split_permille": sp + [0] * (7 - len(sp))}
            assert g.decompose() == (K, L)
            assert np.array_equal(g.kmaxes(), ref_km)
            assert np.array_equal(g.rows(), ref_rows)
            assert all(np.array_equal(x, y) for x, y in zip(g.skyline(), ref_sky))


def test_bad_settings_rejected(dc, gpu):
    V, s, d = dc.gen_rmat(10, 8, 1)
    with dc.Graph.from_edges(V, s, d) as g:
        for bad in [(0, 1, 64, 0), (1, 9, 64, 0), (1, 1, 48, 0), (1, 1, 8, 0), (1, 1, 64, 1000), (1, 1, 64, -1),
                    (1, 1, 64, [400, 300]), (1, 1, 64, [300, 300]), (1, 1, 64, [0, 300]),
                    (1, 1, 64, [1, 2, 3, 4, 5, 6, 7, 8])]:
            with pytest.raises(dc.DCoreError):
                g.set_tuning(*bad)


def test_autotune(dc, orc, gpu):
    V, s, d = dc.gen_rmat(14, 16, 4)
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    with dc.Graph.from_edges(V, s, d) as g:
        best, ms = g.autotune()
        assert 1 <= best["peel_blocks_per_sm"] <= 6 and 1 <= best["rows_blocks_per_sm"] <= 8
        assert best["peel_chunk"] in (32, 64, 128, 256)
        cuts = [c for c in best["rows_split_permille"] if c]
        assert cuts == sorted(set(cuts)) and len(best["rows_split_permille"]) == 7 and len(cuts) <= 3
        assert all(c % 50 == 0 and 50 <= c <= 900 for c in cuts)
        assert best["rows_split_permille"][len(cuts):] == [0] * (7 - len(cuts))
        assert ms > 0
        assert g.tuning() == best
        info = g.decomp_info()
        assert (info["kmax"], info["lmax"]) == (okm, olm)
        assert np.array_equal(g.kmaxes(), okmaxes)
        assert np.array_equal(g.rows(), orows)


def test_split_rows_with_maintenance(dc, orc, gpu):
    from collections import Counter
    V, s, d = dc.gen_rmat(13, 16, 12)
    u, v, dl = dc.gen_updates(V, s, d, 600, 0.5, 13)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_tuning(2, 2, 64, [150, 250, 450, 700, 850])
        g.decompose()
        i = 0
        for bs in (1, 5, 50, 544):
            g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], 2)
            for a, b, x in zip(u[i:i + bs].tolist(), v[i:i + bs].tolist(), dl[i:i + bs].tolist()):
                cnt[(a, b)] += -1 if x else 1
            i += bs
            es = [(a, b) for (a, b), m in cnt.items() for _ in range(m)]
            okm, olm, okmaxes, orows = orc.dcore(V, np.array([a for a, _ in es], np.uint32),
                                                 np.array([b for _, b in es], np.uint32))
            assert np.array_equal(g.kmaxes(), okmaxes)
            assert np.array_equal(g.rows(), orows)
