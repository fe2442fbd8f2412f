"""Host-side helpers of the benchmark: the per-row peel byte model against a
direct count on a small graph, the final edge set of an update stream, the
seeded serving plan and the --tuning parser."""
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_decomposition_bytes_model(dc, orc):
    V, s, d = dc.gen_rmat(10, 8, 3)
    K, kmaxes = orc.kmax(V, s, d)
    m = bench.decomposition_bytes(V, s, d, kmaxes)
    assert m["B_K"] == 12.0 * len(s) + 16.0 * V
    assert len(m["B_row"]) == K + 1
    deg = np.bincount(s, minlength=V) + np.bincount(d, minlength=V)
    for k in (0, 1, K // 2, K):
        inside = kmaxes >= k
        Vk = inside.sum()
        Dk = deg[inside].sum()
        Ik = (inside[s] & inside[d]).sum()
        assert m["B_row"][k] == 8 * Dk + 16 * Ik + 24 * Vk + 4 * (V - Vk)


def test_final_edges_of_a_stream(dc):
    V, s, d = dc.gen_rmat(9, 4, 2)
    u, v, dl = dc.gen_updates(V, s, d, 2000, 0.5, 9)
    fs, fd = bench._final_edges(s, d, u, v, dl)
    live = set(zip(s.tolist(), d.tolist()))
    for a, b, x in zip(u.tolist(), v.tolist(), dl.tolist()):
        if x:
            live.remove((a, b))
        else:
            live.add((a, b))
    assert set(zip(fs.tolist(), fd.tolist())) == live and len(fs) == len(live)


def test_serve_plan_is_seeded():
    w = bench.WORKLOADS["serve-64"]
    a = bench.serve_plan(w, 0)
    b = bench.serve_plan(w, 0)
    c = bench.serve_plan(w, 1)
    assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1])
    for (t1, g1, s1, r1), (t2, g2, s2, r2) in zip(a[2], b[2]):
        assert np.array_equal(t1, t2) and np.array_equal(g1, g2) and np.array_equal(s1, s2)
    assert not np.array_equal(a[2][0][1], c[2][0][1])
    scales, efs, phases = a
    assert scales.min() >= 16 and scales.max() <= 22 and efs.min() >= 8 and efs.max() <= 32
    for t_arr, gid, size, rate in phases:
        assert (np.diff(t_arr) > 0).all() and size.min() >= 1 and size.max() <= 10_000
        assert gid.max() < 64


def test_parse_tuning():
    import pytest
    assert bench.parse_tuning("3,3,64") == (3, 3, 64, [])
    assert bench.parse_tuning("3,3,64,150,250,450") == (3, 3, 64, [150, 250, 450])
    for bad in ("3,3", "1,2,3,4,5,6,7,8,9,10,11", "a,b,c"):
        with pytest.raises(ValueError):
            bench.parse_tuning(bad)
