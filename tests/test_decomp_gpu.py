"""Engine decomposition against the CPU oracle, bit for bit (integer results).

Both engine methods (incremental rows and one peel per row) are checked on
the reference's golden graph, seeded ER graphs at the C1 size (10k vertices,
100k edges) and R-MAT graphs, plus edge cases."""
import os

import numpy as np
import pytest

from test_oracle_golden import GOLD_KMAX, GOLD_KMAXES, GOLD_LMAX, GOLD_ROWS

pytestmark = pytest.mark.gpu

METHODS = [0, 1]


def _expand_skyline(off, ks, ls, kmaxes, K):
    V = len(kmaxes)
    rows = np.zeros((K + 1, V), np.int32)
    for v in range(V):
        a, b = off[v], off[v + 1]
        for i in range(a, b):
            k0 = ks[i]
            k1 = ks[i + 1] if i + 1 < b else kmaxes[v] + 1
            rows[k0:min(k1, kmaxes[v] + 1), v] = ls[i]
    return rows


def check_against_oracle(dc, orc, V, s, d, method, check_skyline=False):
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    with dc.Graph.from_edges(V, s, d) as g:
        kmax, lmax = g.decompose(method)
        assert (kmax, lmax) == (okm, olm)
        km = g.kmaxes()
        assert np.array_equal(km, okmaxes)
        rows = g.rows()
        assert rows.shape == orows.shape
        bad = np.argwhere(rows != orows)
        assert bad.size == 0, f"{len(bad)} mismatches, first (k, v) = {bad[:5].tolist()}"
        if check_skyline:
            off, ks, ls = g.skyline()
            assert np.array_equal(_expand_skyline(off, ks, ls, km, kmax), orows)
        return g.decomp_info()


@pytest.mark.parametrize("method", METHODS)
def test_golden_digraph(dc, gpu, golden_dir, tmp_path, method):
    with dc.Graph.load(os.path.join(golden_dir, "digraph")) as g:
        kmax, lmax = g.decompose(method)
        assert (kmax, lmax) == (GOLD_KMAX, GOLD_LMAX)
        assert g.kmaxes().tolist() == GOLD_KMAXES
        assert g.rows().tolist() == GOLD_ROWS
        out = tmp_path / "digraph.decomp"
        g.write_decomp(str(out))
        assert out.read_bytes() == open(os.path.join(golden_dir, "digraph.decomp"), "rb").read()


def test_golden_binary_load(dc, gpu, golden_dir):
    with dc.Graph.load(os.path.join(golden_dir, "digraph-binary-g=1")) as g:
        assert g.decompose() == (GOLD_KMAX, GOLD_LMAX)
        assert g.rows().tolist() == GOLD_ROWS


@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("method", METHODS)
def test_er_10k(dc, orc, gpu, seed, method):
    s, d = dc.gen_er(10_000, 100_000, seed)
    check_against_oracle(dc, orc, 10_000, s, d, method, check_skyline=(seed == 1))


@pytest.mark.parametrize("scale,ef,seed", [(10, 16, 1), (12, 16, 2), (14, 8, 3), (14, 16, 4)])
@pytest.mark.parametrize("method", METHODS)
def test_rmat_small(dc, orc, gpu, scale, ef, seed, method):
    V, s, d = dc.gen_rmat(scale, ef, seed)
    check_against_oracle(dc, orc, V, s, d, method)


@pytest.mark.parametrize("scale,seed", [(16, 5), (17, 6)])
def test_rmat_medium_incremental(dc, orc, gpu, scale, seed):
    V, s, d = dc.gen_rmat(scale, 16, seed)
    check_against_oracle(dc, orc, V, s, d, 0)


@pytest.mark.parametrize("tuned", [False, True])
def test_rmat20_against_oracle(dc, orc, gpu, tuned):
    """R-MAT 20 (1M vertices, 16M edges): large enough for long cascades in
    the persistent kernels' queues, checked value by value against the
    oracle, with the default launch shapes and with row segments."""
    V, s, d = dc.gen_rmat(20, 16, 7)
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    with dc.Graph.from_edges(V, s, d) as g:
        if tuned:
            g.set_tuning(3, 3, 128, [150, 200, 450])
        assert g.decompose() == (okm, olm)
        assert np.array_equal(g.kmaxes(), okmaxes)
        for k0 in range(0, okm + 1, 64):
            n = min(64, okm + 1 - k0)
            bad = np.argwhere(g.rows(k0, n) != orows[k0:k0 + n])
            assert bad.size == 0, f"rows {k0}..: {len(bad)} mismatches, first {bad[:3].tolist()}"


@pytest.mark.parametrize("method", METHODS)
def test_edge_cases(dc, orc, gpu, method):
    z = np.zeros(0, np.uint32)
    # vertices without edges
    check_against_oracle(dc, orc, 7, z, z, method)
    # one edge, a cycle, a star, multi-edges and self-loops (kept by the engine)
    check_against_oracle(dc, orc, 2, [0], [1], method)
    check_against_oracle(dc, orc, 4, [0, 1, 2, 3], [1, 2, 3, 0], method)
    check_against_oracle(dc, orc, 6, [0] * 5, [1, 2, 3, 4, 5], method)
    check_against_oracle(dc, orc, 3, [0, 0, 1, 1, 2, 2, 0], [1, 1, 2, 2, 0, 0, 0], method)
    # a complete digraph: every vertex in the (n-1, n-1)-core
    n = 12
    s = np.array([u for u in range(n) for v in range(n) if u != v], np.uint32)
    d = np.array([v for u in range(n) for v in range(n) if u != v], np.uint32)
    check_against_oracle(dc, orc, n, s, d, method)


def test_empty_graph(dc, gpu):
    z = np.zeros(0, np.uint32)
    with dc.Graph.from_edges(0, z, z) as g:
        assert g.decompose() == (0, 0)
        assert g.kmaxes().size == 0


def test_bad_vertex_id_rejected(dc, gpu):
    with pytest.raises(dc.DCoreError) as e:
        dc.Graph.from_edges(3, np.array([0, 5], np.uint32), np.array([1, 2], np.uint32))
    assert e.value.code == -1


def test_repeat_decompose_same_handle(dc, orc, gpu):
    s, d = dc.gen_er(2000, 20000, 9)
    okm, olm, okmaxes, orows = orc.dcore(2000, s, d)
    with dc.Graph.from_edges(2000, s, d) as g:
        for method in (0, 1, 0):
            assert g.decompose(method) == (okm, olm)
            assert np.array_equal(g.rows(), orows)


def test_rows_partial_and_device_copy(dc, orc, gpu):
    V, s, d = dc.gen_rmat(12, 16, 11)
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    with dc.Graph.from_edges(V, s, d) as g:
        g.decompose()
        assert np.array_equal(g.rows(3, 5), orows[3:8])
        g.materialize_rows()
        assert np.array_equal(g.rows(), orows)
        g.release_rows()
        assert np.array_equal(g.rows(okm, 1), orows[okm:okm + 1])
