"""C-ABI library: loads without a GPU, exports every declared symbol, host-only
entry points work, compute entry points fail loudly without a device."""
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    names = set()
    for f in os.listdir(os.path.join(ROOT, "include")):
        if f.endswith(".h"):
            txt = open(os.path.join(ROOT, "include", f)).read()
            txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
            names |= set(re.findall(r"\b(dc_[a-z0-9_]+)\s*\(", txt))
    return sorted(names)


def test_library_exports_every_declared_symbol(dc):
    import ctypes
    L = ctypes.CDLL(dc.LIB_PATH)
    declared = _declared()
    assert len(declared) >= 30
    missing = [n for n in declared if not hasattr(L, n)]
    assert not missing, missing


def test_binding_covers_header(dc):
    # every declared function has a ctypes signature in the binding
    missing = [n for n in _declared() if n not in dc.SIGNATURES]
    assert not missing, missing


def test_version_and_error_string(dc):
    assert b"sm_100a" in dc.lib().dc_version()
    assert isinstance(dc.last_error(), str)


def test_er_generator(dc):
    s, d = dc.gen_er(10_000, 100_000, 1)
    assert len(s) == 100_000
    assert (s != d).all()
    keys = s.astype(np.uint64) << 32 | d
    assert (np.diff(keys.astype(np.int64)) > 0).all()  # sorted, unique
    s2, d2 = dc.gen_er(10_000, 100_000, 1)
    assert np.array_equal(s, s2) and np.array_equal(d, d2)
    s3, _ = dc.gen_er(10_000, 100_000, 2)
    assert not np.array_equal(s, s3)


def test_er_generator_limits(dc):
    with pytest.raises(dc.DCoreError):
        dc.gen_er(3, 7, 1)  # more than n*(n-1) edges
    s, d = dc.gen_er(3, 6, 1)  # the complete digraph
    assert sorted(zip(s.tolist(), d.tolist())) == [(0, 1), (0, 2), (1, 0), (1, 2), (2, 0), (2, 1)]


def test_rmat_generator(dc):
    V, s, d = dc.gen_rmat(14, 16, 3)
    assert V == 1 << 14
    assert len(s) < 16 << 14 and len(s) > (16 << 14) * 0.6
    assert (s != d).all() and s.max() < V and d.max() < V
    keys = s.astype(np.uint64) << 32 | d
    assert (np.diff(keys.astype(np.int64)) > 0).all()
    V2, s2, d2 = dc.gen_rmat(14, 16, 3)
    assert np.array_equal(s, s2) and np.array_equal(d, d2)
    # skew: R-MAT has hubs far above the mean degree
    deg = np.bincount(s, minlength=V)
    assert deg.max() > 20 * deg.mean()


def test_no_device_fails_loudly(dc):
    if dc.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(dc.DCoreError) as e:
        dc.Graph.from_edges(3, np.array([0, 1], np.uint32), np.array([1, 2], np.uint32))
    assert e.value.code == -9


def test_server_without_device_fails_loudly(dc):
    if dc.device_count() > 0:
        pytest.skip("a CUDA device is present")
    with pytest.raises(dc.DCoreError) as e:
        dc.Server(1 << 30)
    assert e.value.code == -9


def _replay(s, d, u, v, dl):
    live = set(zip(s.tolist(), d.tolist()))
    for a, b, x in zip(u.tolist(), v.tolist(), dl.tolist()):
        assert a != b
        if x:
            assert (a, b) in live
            live.remove((a, b))
        else:
            assert (a, b) not in live
            live.add((a, b))
    return live


@pytest.mark.parametrize("frac", [0.0, 0.5, 0.6, 1.0])
def test_update_stream_valid_in_sequence(dc, frac):
    V, s, d = dc.gen_rmat(10, 4, 2)
    u, v, dl = dc.gen_updates(V, s, d, 3000, frac, 7)
    _replay(s, d, u, v, dl)
    if 0 < frac < 1:
        assert abs(1 - dl.mean() - frac) < 0.05
    if frac == 1.0:
        assert not dl.any()  # inserts only
    if frac == 0.0:
        assert dl.all()  # deletes only
    u2, v2, dl2 = dc.gen_updates(V, s, d, 3000, frac, 7)
    assert np.array_equal(u, u2) and np.array_equal(v, v2) and np.array_equal(dl, dl2)


def test_hot_update_stream(dc):
    V, s, d = dc.gen_rmat(12, 8, 3)
    od = np.bincount(s, minlength=V)
    hot = np.argsort(-od, kind="stable")[:V // 100].astype(np.uint32)
    n = 4000
    op_hot = np.zeros(n, np.uint8)
    op_hot[1000:1400] = 1
    op_hot[3000:3100] = 1
    u, v, dl = dc.gen_updates_hot(V, s, d, n, 0.6, 11, hot, op_hot)
    _replay(s, d, u, v, dl)
    assert np.isin(u[op_hot == 1], hot).all()
    assert np.isin(u[op_hot == 0], hot).mean() < 0.5
    # without hot operations it is the plain stream
    u0, v0, dl0 = dc.gen_updates(V, s, d, 1000, 0.6, 11)
    assert np.array_equal(u0, u[:1000]) and np.array_equal(dl0, dl[:1000])
