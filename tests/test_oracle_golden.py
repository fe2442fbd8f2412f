"""The CPU oracle against the reference's known-answer decomposition and
against its own literal restatement of the reference pass."""
import os

import numpy as np
import pytest

# dataset/digraph.decomp decoded as int32 (kmax, lmax, kmaxes[8], rows[4][8])
GOLD_KMAX = 3
GOLD_LMAX = 3
GOLD_KMAXES = [2, 3, 3, 2, 3, 3, 3, 3]
GOLD_ROWS = [[2, 2, 3, 2, 3, 3, 2, 3], [2, 2, 3, 2, 3, 3, 2, 3], [2, 2, 3, 2, 3, 3, 2, 3], [0, 1, 3, 0, 3, 3, 1, 3]]


def test_golden_file_decodes_to_known_values(golden_dir):
    raw = np.fromfile(os.path.join(golden_dir, "digraph.decomp"), dtype=np.int32)
    assert raw[0] == GOLD_KMAX and raw[1] == GOLD_LMAX
    assert raw[2:10].tolist() == GOLD_KMAXES
    assert raw[10:].reshape(4, 8).tolist() == GOLD_ROWS


@pytest.mark.parametrize("method", ["bz", "levels"])
def test_oracle_matches_golden(dc, orc, golden_dir, method):
    V, s, d = dc.read_text_edges(os.path.join(golden_dir, "digraph"))
    assert V == 8 and len(s) == 26
    f = orc.dcore if method == "bz" else orc.dcore_levels
    kmax, lmax, kmaxes, rows = f(V, s, d)
    assert kmax == GOLD_KMAX and lmax == GOLD_LMAX
    assert kmaxes.tolist() == GOLD_KMAXES
    assert rows.tolist() == GOLD_ROWS


def _brute_force(V, s, d):
    """(k,l)-core numbers by direct fixpoint of the core definition."""
    s = np.asarray(s)
    d = np.asarray(d)
    kmaxes = np.zeros(V, np.int32)
    # (k, 0)-cores
    k = 0
    alive = np.ones(V, bool)
    while alive.any():
        cur = alive.copy()
        while True:
            m = cur[s] & cur[d]
            indeg = np.bincount(d[m], minlength=V)
            nxt = cur & (indeg >= k)
            if (nxt == cur).all():
                break
            cur = nxt
        kmaxes[cur] = k
        if not cur.any():
            break
        alive = cur
        k += 1
    K = int(kmaxes.max()) if V else 0
    rows = np.zeros((K + 1, V), np.int32)
    for kk in range(K + 1):
        l = 0
        cur = kmaxes >= kk
        while cur.any():
            c2 = cur.copy()
            while True:
                m = c2[s] & c2[d]
                indeg = np.bincount(d[m], minlength=V)
                outdeg = np.bincount(s[m], minlength=V)
                nxt = c2 & (indeg >= kk) & (outdeg >= l)
                if (nxt == c2).all():
                    break
                c2 = nxt
            rows[kk][c2] = l
            if not c2.any():
                break
            cur = c2
            l += 1
    return K, kmaxes, rows


@pytest.mark.parametrize("seed", [1, 2, 3, 4])
def test_oracle_variants_agree_with_brute_force(dc, orc, seed):
    rng = np.random.default_rng(seed)
    V = 40
    m = 180
    s = rng.integers(0, V, m).astype(np.uint32)
    d = rng.integers(0, V, m).astype(np.uint32)
    keep = s != d
    s, d = s[keep], d[keep]  # duplicates kept on purpose (multi-edges)
    K, kb, rb = _brute_force(V, s, d)
    for f in (orc.dcore, orc.dcore_levels):
        kmax, lmax, kmaxes, rows = f(V, s, d)
        assert kmax == K
        assert np.array_equal(kmaxes, kb)
        assert np.array_equal(rows, rb)
        assert lmax == int(rb.max())


@pytest.mark.parametrize("seed", [1, 2, 3])
def test_oracle_bz_equals_levels_er(dc, orc, seed):
    s, d = dc.gen_er(600, 6000, seed)
    a = orc.dcore(600, s, d)
    b = orc.dcore_levels(600, s, d)
    assert a[0] == b[0] and a[1] == b[1]
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])


def test_oracle_bz_equals_levels_rmat(dc, orc):
    V, s, d = dc.gen_rmat(11, 8, 7)
    a = orc.dcore(V, s, d)
    b = orc.dcore_levels(V, s, d)
    assert a[0] == b[0] and a[1] == b[1]
    assert np.array_equal(a[2], b[2]) and np.array_equal(a[3], b[3])


def test_oracle_edge_cases(orc):
    # no edges: every vertex has kmax 0 and row 0 all zero
    km, lm, kmaxes, rows = orc.dcore(5, np.zeros(0, np.uint32), np.zeros(0, np.uint32))
    assert km == 0 and lm == 0 and kmaxes.tolist() == [0] * 5 and rows.tolist() == [[0] * 5]
    # a directed 3-cycle: every vertex in the (1,1)-core
    km, lm, kmaxes, rows = orc.dcore(3, [0, 1, 2], [1, 2, 0])
    assert km == 1 and lm == 1 and rows.tolist() == [[1, 1, 1], [1, 1, 1]]
    # the literal pass returns -1 for an empty vertex set, like KListInplace
    lvl, _ = orc.peel_levels(0, [], [], 0, 0)
    assert lvl == -1


def test_kedge_batches_restatement(orc):
    # roots: endpoint with larger kmax (ties: target); bucket by root kmax
    kmaxes = np.array([0, 1, 1, 2, 2, 0], np.int32)
    frm = np.array([0, 1, 3, 2, 0, 5], np.uint32)
    to = np.array([1, 2, 4, 1, 2, 1], np.uint32)
    nb, batch_of = orc.kedge_batches(6, kmaxes, frm, to)
    # roots: 1 (k1), 2 (k1, tie->to), 4 (k2, tie->to), 1 (k1, tie->to), 2 (k1), 1 (k1)
    # bucket k1 in input order: e0(r1) e1(r2) e3(r1) e4(r2) e5(r1)
    #   pass 1: e0, e1   pass 2: e3, e4   pass 3: e5
    # bucket k2: e2
    assert nb == 4
    assert batch_of.tolist() == [0, 0, 3, 1, 1, 2]
