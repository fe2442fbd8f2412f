"""Batch maintenance against full recomputation (the reference's own test
criterion: main.cu:2116-2143 compares maintained kmaxes/lmaxes with
checkDCore on the updated graph).  Integer results, compared exactly."""
from collections import Counter

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

METHODS = [1, 2]  # DC_MAINT_LOCAL, DC_MAINT_REPEEL


def _edges(cnt):
    s, d = [], []
    for (a, b), m in cnt.items():
        s += [a] * m
        d += [b] * m
    return np.array(s, np.uint32), np.array(d, np.uint32)


def _apply(cnt, u, v, dl):
    for a, b, x in zip(u.tolist(), v.tolist(), dl.tolist()):
        if x:
            cnt[(a, b)] -= 1
            assert cnt[(a, b)] >= 0
            if cnt[(a, b)] == 0:
                del cnt[(a, b)]
        else:
            cnt[(a, b)] += 1


def _check(orc, g, V, cnt):
    s, d = _edges(cnt)
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    info = g.decomp_info()
    assert (info["kmax"], info["lmax"]) == (okm, olm)
    assert np.array_equal(g.kmaxes(), okmaxes)
    rows = g.rows()
    bad = np.argwhere(rows != orows)
    assert bad.size == 0, f"{len(bad)} mismatches, first (k, v) = {bad[:5].tolist()}"


@pytest.mark.parametrize("repair", [2, 1, 0])
@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("scale,seed", [(11, 5), (13, 6)])
def test_mixed_stream_matches_recompute(dc, orc, gpu, method, scale, seed, repair):
    V, s, d = dc.gen_rmat(scale, 8, seed)
    u, v, dl = dc.gen_updates(V, s, d, 700, 0.5, seed + 100)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_row_repair(repair)
        g.decompose()
        i = 0
        for bs in [1, 1, 2, 5, 20, 100, 571]:
            st = g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], method)
            assert st["method"] == method
            _apply(cnt, u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            _check(orc, g, V, cnt)
            i += bs


def test_rmat20_mixed_batches_against_oracle(dc, orc, gpu):
    """R-MAT 20 (1M vertices) with a mixed stream in batches of 10,000, 100
    and 1 under the engine's own method choice and row repair: after each
    batch kmaxes and every row equal the oracle's decomposition of the
    updated graph."""
    V, s, d = dc.gen_rmat(20, 16, 12)
    u, v, dl = dc.gen_updates(V, s, d, 10_101, 0.5, 77)
    base = (s.astype(np.uint64) << np.uint64(32)) | d
    with dc.Graph.from_edges(V, s, d, gap_min=2, gap_div=16) as g:
        g.decompose()
        i = 0
        for bs in (10_000, 100, 1):
            g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            i += bs
            # the edge set after the first i operations (a valid stream:
            # deletions remove present edges, insertions add absent ones)
            ops = (u[:i].astype(np.uint64) << np.uint64(32)) | v[:i]
            keys, inv = np.unique(np.concatenate([base, ops]), return_inverse=True)
            mult = np.bincount(inv, weights=np.concatenate([np.ones(len(base)), np.where(dl[:i] == 1, -1.0, 1.0)]),
                               minlength=len(keys))
            live = keys[mult > 0]
            fs, fd = (live >> np.uint64(32)).astype(np.uint32), (live & np.uint64(0xFFFFFFFF)).astype(np.uint32)
            okm, olm, okmaxes, orows = orc.dcore(V, fs, fd)
            info = g.decomp_info()
            assert (info["kmax"], info["lmax"]) == (okm, olm)
            assert np.array_equal(g.kmaxes(), okmaxes)
            for k0 in range(0, okm + 1, 64):
                n = min(64, okm + 1 - k0)
                assert np.array_equal(g.rows(k0, n), orows[k0:k0 + n]), (bs, k0)


@pytest.mark.parametrize("method", METHODS)
def test_er10k_single_inserts_and_deletes(dc, orc, gpu, method):
    s, d = dc.gen_er(10_000, 100_000, 2)
    u, v, dl = dc.gen_updates(10_000, s, d, 40, 0.5, 9)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    with dc.Graph.from_edges(10_000, s, d) as g:
        g.decompose()
        for i in range(len(u)):
            g.maintain(u[i:i + 1], v[i:i + 1], dl[i:i + 1], method)
            _apply(cnt, u[i:i + 1], v[i:i + 1], dl[i:i + 1])
            if i % 8 == 7:
                _check(orc, g, 10_000, cnt)
        _check(orc, g, 10_000, cnt)


@pytest.mark.parametrize("method", METHODS)
def test_insert_only_and_delete_only_batches(dc, orc, gpu, method):
    V, s, d = dc.gen_rmat(12, 8, 8)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    u, v, dl = dc.gen_updates(V, s, d, 400, 1.0, 3)  # inserts only
    with dc.Graph.from_edges(V, s, d) as g:
        g.decompose()
        g.maintain(u, v, dl, method)
        _apply(cnt, u, v, dl)
        _check(orc, g, V, cnt)
        # delete 300 present edges in one batch
        es = list(cnt.keys())[:300]
        du = np.array([a for a, _ in es], np.uint32)
        dv = np.array([b for _, b in es], np.uint32)
        g.maintain(du, dv, np.ones(len(du), np.uint8), method)
        _apply(cnt, du, dv, np.ones(len(du), np.uint8))
        _check(orc, g, V, cnt)


def test_delete_missing_edge_rejected_graph_unchanged(dc, orc, gpu):
    s, d = dc.gen_er(500, 3000, 4)
    present = set(zip(s.tolist(), d.tolist()))
    absent = [(a, b) for a in range(500) for b in range(500) if a != b and (a, b) not in present][:2]
    ins, miss = absent
    with dc.Graph.from_edges(500, s, d) as g:
        g.decompose()
        before = g.rows().copy()
        # a valid insertion plus a deletion of an absent edge: nothing is applied
        with pytest.raises(dc.DCoreError) as e:
            g.maintain(np.array([ins[0], miss[0]], np.uint32), np.array([ins[1], miss[1]], np.uint32),
                       np.array([0, 1], np.uint8))
        assert e.value.code == -7
        g2s, g2d = g.edges()
        assert sorted(zip(g2s.tolist(), g2d.tolist())) == sorted(present)
        g.decompose()
        assert np.array_equal(g.rows(), before)


def test_net_zero_and_multi_edges(dc, orc, gpu):
    s, d = dc.gen_er(300, 2000, 6)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    a, b = int(s[0]), int(d[0])  # present edge
    with dc.Graph.from_edges(300, s, d) as g:
        g.decompose()
        # delete and re-insert the same edge, insert a duplicate of another
        u = np.array([a, a, s[1], s[1]], np.uint32)
        v = np.array([b, b, d[1], d[1]], np.uint32)
        dl = np.array([1, 0, 0, 0], np.uint8)
        st = g.maintain(u, v, dl)
        assert st["deleted"] == 0 and st["inserted"] == 2
        _apply(cnt, u, v, dl)
        _check(orc, g, 300, cnt)


@pytest.mark.parametrize("method", METHODS)
def test_slack_overflow_rebuilds_store(dc, orc, gpu, method):
    V, s, d = dc.gen_rmat(10, 8, 12)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    present = set(cnt)
    hub = int(np.bincount(s, minlength=V).argmax())
    targets = [t for t in range(V) if t != hub and (hub, t) not in present][:40]
    u = np.full(len(targets), hub, np.uint32)
    v = np.array(targets, np.uint32)
    with dc.Graph.from_edges(V, s, d, gap_min=1) as g:
        g.decompose()
        st = g.maintain(u, v, np.zeros(len(u), np.uint8), method)
        assert st["rebuilt"] == 1
        _apply(cnt, u, v, np.zeros(len(u), np.uint8))
        _check(orc, g, V, cnt)
        # the rebuilt store takes further updates
        st = g.maintain(v[:5], u[:5], np.zeros(5, np.uint8), method)
        _apply(cnt, v[:5], u[:5], np.zeros(5, np.uint8))
        _check(orc, g, V, cnt)


def test_maintain_before_decompose_and_auto(dc, orc, gpu):
    V, s, d = dc.gen_rmat(11, 8, 13)
    u, v, dl = dc.gen_updates(V, s, d, 50, 0.5, 14)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    with dc.Graph.from_edges(V, s, d) as g:
        st = g.maintain(u, v, dl, 0)  # decomposes first, scheduler picks
        assert st["method"] in (1, 2)
        _apply(cnt, u, v, dl)
        _check(orc, g, V, cnt)


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("scale,ef,seed", [(12, 16, 21), (14, 8, 22)])
def test_deletion_stream_local_row_repair(dc, orc, gpu, method, scale, ef, seed):
    # deletions only: rows are repaired in place from their old values
    V, s, d = dc.gen_rmat(scale, ef, seed)
    sizes = [1, 1, 2, 3, 10, 50, 200, 1000]
    u, v, dl = dc.gen_updates(V, s, d, sum(sizes), 0.0, seed + 7)
    assert dl.all()
    cnt = Counter(zip(s.tolist(), d.tolist()))
    local = 0
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_row_repair(2)  # in place whenever the deletions fit
        g.decompose()
        i = 0
        for bs in sizes:
            st = g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], method)
            local += st["rows_local"]
            _apply(cnt, u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            _check(orc, g, V, cnt)
            i += bs
    assert local >= len(sizes) // 2  # the in-place path ran


@pytest.mark.parametrize("seed", range(1, 13))
def test_randomized_deletion_heavy_streams(dc, orc, gpu, seed):
    # random graphs, batch sizes and methods, mostly deletions: every batch
    # leaves kmaxes and every row equal to a recomputation
    rng = np.random.default_rng(seed)
    V, s, d = dc.gen_rmat(int(rng.integers(10, 14)), int(rng.choice([8, 16])), seed)
    sizes = [int(x) for x in rng.integers(1, 700, 3)]
    u, v, dl = dc.gen_updates(V, s, d, sum(sizes), float(rng.choice([0.0, 0.3])), seed + 50)
    method = int(rng.choice(METHODS))
    cnt = Counter(zip(s.tolist(), d.tolist()))
    with dc.Graph.from_edges(V, s, d) as g:
        g.decompose()
        i = 0
        for bs in sizes:
            g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], method)
            _apply(cnt, u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            _check(orc, g, V, cnt)
            i += bs


@pytest.mark.parametrize("method", METHODS)
@pytest.mark.parametrize("scale,ef,seed", [(12, 16, 31), (14, 8, 32)])
def test_insertion_stream_local_row_repair(dc, orc, gpu, method, scale, ef, seed):
    # insertions only: rows are repaired in place row after row (values can
    # only rise; the region grows from the inserted edges and the vertices
    # that joined C_k), every batch checked against a recomputation
    V, s, d = dc.gen_rmat(scale, ef, seed)
    sizes = [1, 1, 2, 3, 10, 50, 200, 1000]
    u, v, dl = dc.gen_updates(V, s, d, sum(sizes), 1.0, seed + 7)
    assert not dl.any()
    cnt = Counter(zip(s.tolist(), d.tolist()))
    local = 0
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_row_repair(2)  # in place whenever the insertions fit
        g.decompose()
        i = 0
        for bs in sizes:
            st = g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], method)
            local += (st["rows_local"] >> 1) & 1
            _apply(cnt, u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            _check(orc, g, V, cnt)
            i += bs
    assert local >= len(sizes) // 2  # the in-place path ran


def test_insertions_into_the_dense_core(dc, orc, gpu):
    # edges between high-kmax vertices: kmax rises, vertices join C_k for
    # high k, and the in-degree condition of whole rows moves
    V, s, d = dc.gen_rmat(12, 16, 41)
    cnt = Counter(zip(s.tolist(), d.tolist()))
    km, kmaxes = orc.kmax(V, s, d)
    top = np.argsort(-kmaxes, kind="stable")[:400].astype(np.uint32)
    rng = np.random.default_rng(3)
    pairs = []
    while len(pairs) < 60:
        a, b = (int(x) for x in rng.choice(top, 2, replace=False))
        if (a, b) not in cnt and (a, b) not in pairs:
            pairs.append((a, b))
    local = 0
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_row_repair(2)
        g.decompose()
        for i in range(0, len(pairs), 6):
            u = np.array([p[0] for p in pairs[i:i + 6]], np.uint32)
            v = np.array([p[1] for p in pairs[i:i + 6]], np.uint32)
            z = np.zeros(len(u), np.uint8)
            st = g.maintain(u, v, z, 1)
            local += (st["rows_local"] >> 1) & 1
            _apply(cnt, u, v, z)
            _check(orc, g, V, cnt)
    assert local > 0


@pytest.mark.parametrize("seed", range(1, 13))
def test_randomized_insertion_heavy_streams(dc, orc, gpu, seed):
    # random graphs, batch sizes, methods and row modes, mostly insertions
    rng = np.random.default_rng(100 + seed)
    V, s, d = dc.gen_rmat(int(rng.integers(10, 14)), int(rng.choice([8, 16])), seed)
    sizes = [int(x) for x in rng.integers(1, 400, 4)]
    u, v, dl = dc.gen_updates(V, s, d, sum(sizes), float(rng.choice([1.0, 0.7])), seed + 60)
    method = int(rng.choice(METHODS))
    cnt = Counter(zip(s.tolist(), d.tolist()))
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_row_repair(int(rng.choice([1, 2])))
        g.decompose()
        i = 0
        for bs in sizes:
            g.maintain(u[i:i + bs], v[i:i + bs], dl[i:i + bs], method)
            _apply(cnt, u[i:i + bs], v[i:i + bs], dl[i:i + bs])
            _check(orc, g, V, cnt)
            i += bs
