"""Host-side helpers of the benchmark: the byte models against direct counts
on small graphs, the shared config of both arms, the reference arm's
isolation from the engine library, the final edge set of an update stream,
the seeded serving plan and the --tuning parser."""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

import bench  # noqa: E402


def test_refinement_bytes_model(orc):
    """The row-refinement byte model against a direct count: every value
    that changes from row k-1 to row k reads its lists' entries inside C_k."""
    V, s, d = orc.gen_rmat(10, 8, 3)
    K, L, kmaxes, rows = orc.dcore(V, s, d)
    b, changes, entries = bench.refinement_bytes(V, s, d, kmaxes, rows)
    n_ch = n_ent = 0
    for k in range(1, K + 1):
        inside = kmaxes >= k
        for v in np.nonzero(inside & (rows[k] != rows[k - 1]))[0]:
            n_ch += 1
            n_ent += int(inside[d[s == v]].sum() + inside[s[d == v]].sum())
    assert (changes, entries) == (n_ch, n_ent)
    assert b == 8.0 * n_ent + 20.0 * n_ch + 4.0 * (V - np.count_nonzero(kmaxes == K))


def test_peel_bytes_model(orc):
    V, s, d = orc.gen_rmat(9, 8, 2)
    E = len(s)
    assert bench.peel_bytes(V, s, d, None) == (12.0 * E + 16.0 * V) + (16.0 * E + 16.0 * E + 24.0 * V)


def test_decomp_config_is_the_same_for_both_arms():
    """The reference arm and the engine arm print one config for a workload."""
    class A:
        workload = "decomp-rmat22"
    w = bench.WORKLOADS["decomp-rmat22"]
    a = bench.decomp_config(A, w, 4194304, 65245102, 592, 591, 1)
    b = bench.decomp_config(A, w, 4194304, 65245102, 592, 591, 1)
    assert a == b and a["workload"] == "decomp-rmat22" and a["E"] == 65245102


def test_reference_arm_does_not_load_the_engine(tmp_path):
    """bench.py --impl reference runs the oracle alone: the engine library
    must not be loaded by that process."""
    import subprocess
    code = ("import sys, json; sys.argv=['bench.py','--impl','reference','--workload','decomp-er10k',"
            "'--steps','1','--warmup','1']; import bench; bench.main(); "
            "print(json.dumps([m for m in open('/proc/self/maps').read().split() if m.endswith('.so')]))")
    p = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=300)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = p.stdout.strip().splitlines()
    line = json.loads(lines[0])
    maps = json.loads(lines[-1])
    assert line["impl"] == "reference" and line["config"]["E"] == 100_000 and line["steps"] == 1
    assert not any("libdcore_b200" in m for m in maps)
    assert any("liboracle" in m for m in maps)


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
