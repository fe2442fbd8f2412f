"""Maintenance batches run as one captured CUDA graph (dc_set_captured_batches):
every batch leaves the decomposition equal to the oracle's recomputation and
to the host-driven path's result, the device-side branches (missing
deletion, list without free slots, repair not worth it) end where the
host-driven batch ends.  Integer results, compared exactly."""
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


def _check(orc, g, V, cnt):
    s = np.array([a for (a, b), m in cnt.items() for _ in range(m)], np.uint32)
    d = np.array([b for (a, b), m in cnt.items() for _ in range(m)], np.uint32)
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    info = g.decomp_info()
    assert (info["kmax"], info["lmax"]) == (okm, olm)
    assert np.array_equal(g.kmaxes(), okmaxes)
    assert np.array_equal(g.rows(), orows)


@pytest.mark.parametrize("mode", [1, 2, 3])
@pytest.mark.parametrize("frac", [0.0, 1.0])
def test_one_kind_batches_run_captured(dc, orc, gpu, mode, frac):
    V, s, d = dc.gen_rmat(12, 16, 51)
    sizes = [1, 1, 2, 3, 8, 20, 64, 200]
    u, v, dl = dc.gen_updates(V, s, d, sum(sizes), frac, 52)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    captured = 0
    with dc.Graph.from_edges(V, s, d, gap_min=8, gap_div=8) as g:  # room for every insertion
        g.set_row_repair(mode)
        g.decompose()
        i = 0
        for bs in sizes:
            st = g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], 1)
            captured += st["captured"]
            _apply(cnt, u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            _check(orc, g, V, cnt)
            i += bs
    # mode 1 captures batches of at most 64 net updates, modes 2 and 3 all of these
    assert captured >= (7 if mode == 1 else len(sizes))


def test_captured_equals_host_driven_on_mixed_stream(dc, orc, gpu):
    V, s, d = dc.gen_rmat(13, 8, 53)
    sizes = [1, 1, 1, 2, 4, 10, 30, 60, 1, 1]
    u, v, dl = dc.gen_updates(V, s, d, sum(sizes), 0.5, 54)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    with dc.Graph.from_edges(V, s, d) as a, dc.Graph.from_edges(V, s, d) as b:
        b.set_captured_batches(False)
        for g in (a, b):
            g.set_row_repair(3)
            g.decompose()
        n_cap = 0
        i = 0
        for bs in sizes:
            sa = a.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], 1)
            sb = b.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], 1)
            assert sb["captured"] == 0
            n_cap += sa["captured"]
            assert (sa["kmax"], sa["lmax"]) == (sb["kmax"], sb["lmax"])
            assert np.array_equal(a.kmaxes(), b.kmaxes())
            assert np.array_equal(a.rows(), b.rows())
            _apply(cnt, u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            i += bs
        _check(orc, a, V, cnt)
        assert n_cap >= 4


def test_captured_missing_deletion_leaves_graph_unchanged(dc, orc, gpu):
    s, d = dc.gen_er(400, 3000, 55)
    present = set(zip(s.tolist(), d.tolist()))
    miss = next((x, y) for x in range(400) for y in range(400) if x != y and (x, y) not in present)
    with dc.Graph.from_edges(400, s, d) as g:
        g.decompose()
        before = g.rows().copy()
        with pytest.raises(dc.DCoreError) as e:
            g.maintain(np.array([s[0], miss[0]], np.uint32), np.array([d[0], miss[1]], np.uint32),
                       np.array([1, 1], np.uint8), 1)
        assert e.value.code == -7
        g2s, g2d = g.edges()
        assert sorted(zip(g2s.tolist(), g2d.tolist())) == sorted(present)
        assert np.array_equal(g.rows(), before)
        # the handle keeps working
        st = g.maintain(s[:1], d[:1], np.ones(1, np.uint8), 1)
        assert st["captured"] == 1
        cnt = Counter(present)
        _apply(cnt, s[:1], d[:1], np.ones(1, np.uint8))
        _check(orc, g, 400, cnt)


def test_captured_full_list_falls_back_to_rebuild(dc, orc, gpu):
    V, s, d = dc.gen_rmat(10, 8, 56)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    hub = int(np.bincount(s, minlength=V).argmax())
    targets = [t for t in range(V) if t != hub and (hub, t) not in cnt][:20]
    u = np.full(len(targets), hub, np.uint32)
    v = np.array(targets, np.uint32)
    z = np.zeros(len(u), np.uint8)
    with dc.Graph.from_edges(V, s, d, gap_min=1) as g:
        g.set_row_repair(2)
        g.decompose()
        st = g.maintain(u, v, z, 1)
        assert st["rebuilt"] == 1 and st["captured"] == 0
        _apply(cnt, u, v, z)
        _check(orc, g, V, cnt)


def test_captured_rows_recomputed_when_repair_not_taken(dc, orc, gpu):
    # row mode 1: deletions whose expected repair work is too large are
    # recomputed by the host after the graph (captured, no rows in place)
    V, s, d = dc.gen_rmat(12, 16, 57)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    km, kmaxes = orc.kmax(V, s, d)
    deg = np.bincount(s, minlength=V) + np.bincount(d, minlength=V)
    score = deg.astype(np.int64) * kmaxes
    order = np.argsort(-(score[s] + score[d]), kind="stable")[:40]
    u, v = s[order], d[order]
    dl = np.ones(len(u), np.uint8)
    with dc.Graph.from_edges(V, s, d) as g:
        g.decompose()
        st = g.maintain(u, v, dl, 1)
        assert st["captured"] == 1 and st["rows_local"] == 0
        _apply(cnt, u, v, dl)
        _check(orc, g, V, cnt)
