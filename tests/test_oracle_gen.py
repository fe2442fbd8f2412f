"""The oracle's generators (gen_oracle.c) give exactly the engine's seeded
graphs.  The benchmark's reference arm builds its inputs with them so that it
never loads the engine library; its numbers are only comparable if the graphs
are the same.  Host only: the engine's generators need no GPU."""
import numpy as np
import pytest


@pytest.mark.parametrize("scale,ef,seed", [(1, 4, 1), (8, 8, 2), (12, 16, 3), (15, 16, 1), (17, 8, 5)])
def test_rmat_matches_engine(dc, orc, scale, ef, seed):
    Va, sa, da = orc.gen_rmat(scale, ef, seed)
    Vb, sb, db = dc.gen_rmat(scale, ef, seed)
    assert Va == Vb
    assert np.array_equal(sa, sb) and np.array_equal(da, db)


def test_rmat_other_parameters_match_engine(dc, orc):
    for kw in (dict(permute=False), dict(a=0.25, b=0.25, c=0.25), dict(a=0.45, b=0.15, c=0.15, permute=False)):
        Va, sa, da = orc.gen_rmat(11, 12, 7, **kw)
        Vb, sb, db = dc.gen_rmat(11, 12, 7, **kw)
        assert np.array_equal(sa, sb) and np.array_equal(da, db), kw


@pytest.mark.parametrize("n,m,seed", [(2, 2, 1), (10, 90, 3), (10_000, 100_000, 1), (10_000, 100_000, 2),
                                      (300, 80_000, 9)])
def test_er_matches_engine(dc, orc, n, m, seed):
    sa, da = orc.gen_er(n, m, seed)
    sb, db = dc.gen_er(n, m, seed)
    assert np.array_equal(sa, sb) and np.array_equal(da, db)
