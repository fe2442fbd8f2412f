"""Reference file formats: text graph, -binary-g=N cache, .decomp, .decompCPU.
Host-only code paths, checked byte for byte against the reference's files."""
import os

import numpy as np
import pytest

from test_oracle_golden import GOLD_KMAX, GOLD_KMAXES, GOLD_LMAX, GOLD_ROWS


def _golden_edges(golden_dir):
    lines = open(os.path.join(golden_dir, "digraph")).read().split("\n")[1:]
    pairs = [tuple(map(int, l.split())) for l in lines if l.strip()]
    return pairs


def test_text_reader(dc, golden_dir):
    V, s, d = dc.read_text_edges(os.path.join(golden_dir, "digraph"))
    assert V == 8
    assert list(zip(s.tolist(), d.tolist())) == _golden_edges(golden_dir)


def test_text_reader_prunes_self_loops_and_empty_vertices(dc, tmp_path):
    p = tmp_path / "g"
    p.write_text("# 100\n3 3\n3 7\n7 50\n50 3\n9 9\n")
    V, s, d = dc.read_text_edges(str(p))
    # 9 has only a self loop -> pruned; 3,7,50 -> 0,1,2
    assert V == 3
    assert list(zip(s.tolist(), d.tolist())) == [(0, 1), (1, 2), (2, 0)]
    V2, s2, d2 = dc.read_text_edges(str(p), prune=False)
    assert V2 == 100 and list(zip(s2.tolist(), d2.tolist())) == [(3, 7), (7, 50), (50, 3)]


def test_text_reader_keeps_duplicates(dc, tmp_path):
    p = tmp_path / "g"
    p.write_text("# 2\n0 1\n0 1\n1 0\n")
    V, s, d = dc.read_text_edges(str(p))
    assert V == 2 and len(s) == 3


def test_text_reader_errors(dc, tmp_path):
    with pytest.raises(dc.DCoreError) as e:
        dc.read_text_edges(str(tmp_path / "missing"))
    assert e.value.code == -4
    p = tmp_path / "bad"
    p.write_text("# 3\n0 1\nfoo bar\n")
    with pytest.raises(dc.DCoreError) as e:
        dc.read_text_edges(str(p))
    assert e.value.code == -1
    p.write_text("")
    with pytest.raises(dc.DCoreError):
        dc.read_text_edges(str(p))


def test_binary_writer_reproduces_reference_cache(dc, golden_dir, tmp_path):
    V, s, d = dc.read_text_edges(os.path.join(golden_dir, "digraph"))
    out = tmp_path / "digraph-binary-g=1"
    dc.write_binary_edges(str(out), V, s, d, gap=1)
    assert out.read_bytes() == open(os.path.join(golden_dir, "digraph-binary-g=1"), "rb").read()


def test_binary_reader(dc, golden_dir):
    V, s, d = dc.read_binary_edges(os.path.join(golden_dir, "digraph-binary-g=1"))
    assert V == 8 and len(s) == 26
    assert sorted(zip(s.tolist(), d.tolist())) == sorted(_golden_edges(golden_dir))


def test_binary_layout_pinned(golden_dir):
    raw = np.fromfile(os.path.join(golden_dir, "digraph-binary-g=1"), dtype=np.uint32)
    V, E = raw[0], raw[1]
    assert (V, E) == (8, 26)
    in_off = raw[2 + 2 * V: 2 + 3 * V + 1]
    assert in_off.tolist() == [0, 3, 8, 14, 17, 21, 26, 30, 34]


def test_binary_reader_rejects_truncated(dc, golden_dir, tmp_path):
    data = open(os.path.join(golden_dir, "digraph-binary-g=1"), "rb").read()
    for cut in (4, 40, len(data) - 4):
        p = tmp_path / f"t{cut}-binary-g=1"
        p.write_bytes(data[:cut])
        with pytest.raises(dc.DCoreError) as e:
            dc.read_binary_edges(str(p))
        assert e.value.code == -1


def test_binary_roundtrip_gap(dc, tmp_path):
    s, d = dc.gen_er(300, 2000, 5)
    for gap in (0, 1, 4):
        p = tmp_path / f"g-binary-g={gap}"
        dc.write_binary_edges(str(p), 300, s, d, gap=gap)
        V, s2, d2 = dc.read_binary_edges(str(p))
        assert V == 300
        assert sorted(zip(s2.tolist(), d2.tolist())) == sorted(zip(s.tolist(), d.tolist()))


def test_decomp_writer_reproduces_reference_file(dc, golden_dir, tmp_path):
    out = tmp_path / "digraph.decomp"
    rows = np.array(GOLD_ROWS, np.int32)
    dc.write_decomp_file(str(out), GOLD_KMAX, GOLD_LMAX, np.array(GOLD_KMAXES, np.int32), rows)
    assert out.read_bytes() == open(os.path.join(golden_dir, "digraph.decomp"), "rb").read()
    km, lm, kmaxes, rows2 = dc.read_decomp_file(os.path.join(golden_dir, "digraph.decomp"), 8)
    assert (km, lm) == (GOLD_KMAX, GOLD_LMAX)
    assert kmaxes.tolist() == GOLD_KMAXES and rows2.tolist() == GOLD_ROWS


def test_decomp_reader_rejects_wrong_size(dc, golden_dir):
    with pytest.raises(dc.DCoreError):
        dc.read_decomp_file(os.path.join(golden_dir, "digraph.decomp"), 9)


def test_decomp_cpu_format(dc, tmp_path):
    out = tmp_path / "x.decompCPU"
    dc.write_decomp_cpu_file(str(out), np.array(GOLD_KMAXES, np.int32), np.array(GOLD_ROWS, np.int32))
    lines = out.read_text().split("\n")
    assert lines[0] == "8"
    # vertex v lists rows 0..kmax[v]
    assert lines[1] == "2 2 2"          # v0: kmax 2
    assert lines[2] == "2 2 2 1"        # v1: kmax 3
    assert lines[8] == "3 3 3 3"        # v7
    assert not out.read_text().endswith("\n")
