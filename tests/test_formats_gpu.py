"""GPU-side file formats: the text graph parsed on the device
(dc_graph_load_text_device) gives the graph the host parser gives, and the
.decompCPU text formatted on the device (dc_write_decomp_cpu_device) is
byte-identical to the host writer's (writeDecompFileCPU, src/utils.h:110-124)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _sorted_edges(s, d):
    k = (np.asarray(s, np.uint64) << np.uint64(32)) | np.asarray(d, np.uint64)
    return np.sort(k)


def _same_graph(dc, path, prune):
    V, s, d = dc.read_text_edges(path, prune=prune)
    with dc.Graph.load_text_device(path, prune=prune) as g:
        gv, ge = g.info()
        gs, gd = g.edges()
    assert (gv, ge) == (V, len(s))
    assert np.array_equal(_sorted_edges(gs, gd), _sorted_edges(s, d))


@pytest.mark.parametrize("prune", [True, False])
def test_golden_text_parsed_on_device(dc, gpu, golden_dir, prune):
    _same_graph(dc, os.path.join(golden_dir, "digraph"), prune)


@pytest.mark.parametrize("prune", [True, False])
def test_awkward_text_parsed_on_device(dc, gpu, tmp_path, prune):
    """Comments, blank and CRLF lines, tabs, '+' signs, self-loops,
    duplicates, trailing text, sparse ids and no final newline."""
    p = tmp_path / "g"
    p.write_bytes(b"#  1000\n3 7\n\n# a comment\n  7\t50\r\n50 3\n9 9\n+4 +3 extra\n3 7\n\t\n999 3")
    _same_graph(dc, str(p), prune)


@pytest.mark.parametrize("prune", [True, False])
def test_large_text_parsed_on_device(dc, gpu, tmp_path, prune):
    V, s, d = dc.gen_rmat(14, 16, 5)
    rng = np.random.default_rng(1)
    lines = [f"{a} {b}" for a, b in zip(s.tolist(), d.tolist())]
    for i in rng.integers(0, len(lines), 200).tolist():  # self-loops and duplicates sprinkled in
        lines[i] = lines[i] + ("\n%d %d" % (i % V, i % V) if i % 2 else "\n" + lines[i])
    p = tmp_path / "g"
    p.write_text(f"# {V}\n" + "\n".join(lines) + "\n")
    _same_graph(dc, str(p), prune)


def test_malformed_text_rejected_on_device(dc, gpu, tmp_path):
    p = tmp_path / "g"
    p.write_text("# 5\n0 1\n1 x\n2 3\n")
    with pytest.raises(dc.DCoreError) as e:
        dc.Graph.load_text_device(str(p))
    assert e.value.code == -1 and ":3:" in str(e.value)
    q = tmp_path / "h"
    q.write_text("# 5\n0 1\n4294967295 2\n")
    with pytest.raises(dc.DCoreError):
        dc.Graph.load_text_device(str(q))


def test_header_only_text_on_device(dc, gpu, tmp_path):
    p = tmp_path / "g"
    p.write_text("# 6\n")
    _same_graph(dc, str(p), True)
    _same_graph(dc, str(p), False)


@pytest.mark.parametrize("which", ["golden", "er", "rmat", "isolated"])
def test_decomp_cpu_written_on_device(dc, gpu, golden_dir, tmp_path, which):
    if which == "golden":
        g = dc.Graph.load(os.path.join(golden_dir, "digraph"))
    elif which == "er":
        s, d = dc.gen_er(10_000, 100_000, 3)
        g = dc.Graph.from_edges(10_000, s, d)
    elif which == "rmat":
        V, s, d = dc.gen_rmat(14, 16, 6)
        g = dc.Graph.from_edges(V, s, d)
    else:  # vertices without edges (kmax 0, one value per line) and a 2-cycle
        g = dc.Graph.from_edges(9, np.array([3, 4], np.uint32), np.array([4, 3], np.uint32))
    with g:
        g.decompose()
        a, b = tmp_path / "host.decompCPU", tmp_path / "dev.decompCPU"
        g.write_decomp_cpu(str(a))
        g.write_decomp_cpu_device(str(b))
        assert a.read_bytes() == b.read_bytes()
