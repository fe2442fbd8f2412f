"""Parity with the reference itself: its own dcore() (main.cu:197-262), built
from its sources into oracle/_ref/ref_dcore, run on the same graphs as the
engine, results compared exactly (kmax, lmax, kmaxes, every row).  Graphs
stay below V = 1,000,000, the reference's peel-buffer capacity."""
import numpy as np
import pytest

from oracle import ref_gpu

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not ref_gpu.available(),
                                 reason="oracle/_ref/ref_dcore not built (needs the reference sources)")]


def _engine(dc, V, s, d):
    with dc.Graph.from_edges(V, s, d) as g:
        km, lm = g.decompose()
        return km, lm, g.kmaxes(), g.rows()


def _same(dc, V, s, d):
    rk, rl, rkm, rrows, _ = ref_gpu.dcore(V, s, d)
    ek, el, ekm, erows = _engine(dc, V, s, d)
    assert (ek, el) == (rk, rl)
    assert np.array_equal(ekm, rkm)
    assert np.array_equal(erows, rrows)


def test_golden_graph(dc, gpu, golden_dir):
    import os
    V, s, d = dc.read_text_edges(os.path.join(golden_dir, "digraph"))
    _same(dc, V, s, d)


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_er_10k_100k(dc, gpu, seed):
    s, d = dc.gen_er(10_000, 100_000, seed)
    _same(dc, 10_000, s, d)


@pytest.mark.parametrize("scale,ef,seed", [(12, 8, 1), (14, 16, 2), (16, 16, 3)])
def test_rmat(dc, gpu, scale, ef, seed):
    V, s, d = dc.gen_rmat(scale, ef, seed)
    _same(dc, V, s, d)
