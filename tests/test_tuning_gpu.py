"""Launch shapes change speed, never answers: the decomposition under several
peel grids, chunk sizes and row-kernel grids equals the default one, and the
autotuner leaves a valid setting and a full decomposition behind."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

SETTINGS = [(1, 1, 16), (2, 1, 32), (1, 2, 128), (4, 4, 256), (3, 2, 4096)]


def test_settings_give_identical_results(dc, gpu):
    V, s, d = dc.gen_rmat(15, 16, 9)
    with dc.Graph.from_edges(V, s, d) as g:
        K, L = g.decompose()
        ref_km, ref_rows = g.kmaxes(), g.rows()
        for pb, rb, ch in SETTINGS:
            g.set_tuning(pb, rb, ch)
            assert g.tuning() == {"peel_blocks_per_sm": pb, "rows_blocks_per_sm": rb, "peel_chunk": ch}
            assert g.decompose() == (K, L)
            assert np.array_equal(g.kmaxes(), ref_km)
            assert np.array_equal(g.rows(), ref_rows)


def test_bad_settings_rejected(dc, gpu):
    V, s, d = dc.gen_rmat(10, 8, 1)
    with dc.Graph.from_edges(V, s, d) as g:
        for bad in [(0, 1, 64), (1, 9, 64), (1, 1, 48), (1, 1, 8)]:
            with pytest.raises(dc.DCoreError):
                g.set_tuning(*bad)


def test_autotune(dc, orc, gpu):
    V, s, d = dc.gen_rmat(14, 16, 4)
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    with dc.Graph.from_edges(V, s, d) as g:
        best, ms = g.autotune()
        assert 1 <= best["peel_blocks_per_sm"] <= 6 and 1 <= best["rows_blocks_per_sm"] <= 8
        assert best["peel_chunk"] in (32, 64, 128, 256)
        assert ms > 0
        assert g.tuning() == best
        info = g.decomp_info()
        assert (info["kmax"], info["lmax"]) == (okm, olm)
        assert np.array_equal(g.kmaxes(), okmaxes)
        assert np.array_equal(g.rows(), orows)
