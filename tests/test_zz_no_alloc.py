"""The allocation-free kmax entry point (dc_kmax_noalloc).

It exists for callers that cannot let a library call cudaMalloc (code that
owns every device allocation through its own pool, or serving loops that
cannot afford cudaMalloc's device-wide synchronisation).  Its results must
equal those of the regular entry point (dc_decompose + dc_get_kmaxes), also
when two calls run back to back and the second one finds the shared scratch
array still holding the first call's state.  This file sorts last so that a
run stopping at the first failure has run every other test before it.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _csr(V, src, dst):
    """CSC offsets (by target) and CSR offsets + neighbours (by source)."""
    order = np.lexsort((dst, src))
    out_nbr = dst[order].astype(np.uint32)
    out_off = np.zeros(V + 1, np.uint32)
    np.cumsum(np.bincount(src, minlength=V), out=out_off[1:])
    in_off = np.zeros(V + 1, np.uint32)
    np.cumsum(np.bincount(dst, minlength=V), out=in_off[1:])
    return in_off, out_off, out_nbr


def _noalloc_kmax(dc, V, src, dst):
    import torch
    in_off, out_off, out_nbr = _csr(V, src, dst)
    dev = torch.device("cuda", 0)
    t_in = torch.from_numpy(in_off.view(np.int32)).to(dev)
    t_oo = torch.from_numpy(out_off.view(np.int32)).to(dev)
    t_on = torch.from_numpy(np.ascontiguousarray(out_nbr).view(np.int32)).to(dev)
    t_k = torch.full((max(V, 1),), -7, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    kmax_max = ctypes.c_int32(-1)
    torch.cuda.synchronize()
    rc = dc.lib().dc_kmax_noalloc(V, len(src), t_in.data_ptr(), t_oo.data_ptr(), t_on.data_ptr(), t_k.data_ptr(),
                                  ctypes.byref(kmax_max), stream.cuda_stream)
    assert rc == 0, dc.last_error()
    return t_k[:V].cpu().numpy(), kmax_max.value


def _regular_kmax(dc, V, src, dst):
    with dc.Graph.from_edges(V, src, dst) as g:
        kmax, _ = g.decompose()
        return g.kmaxes(), kmax


def test_noalloc_kmax_matches_regular_entry_point_twice_in_a_row(dc, orc, gpu):
    graphs = [dc.gen_rmat(14, 16, 21), dc.gen_rmat(13, 8, 22)]
    s, d = dc.gen_er(10_000, 100_000, 23)
    graphs.append((10_000, s, d))
    for V, src, dst in graphs:
        ref, ref_max = _regular_kmax(dc, V, src, dst)
        o_max, o_kmaxes = orc.kmax(V, src, dst)
        assert o_max == ref_max and np.array_equal(o_kmaxes, ref)
        for _ in range(2):  # back to back: the scratch keeps the previous call's contents
            got, got_max = _noalloc_kmax(dc, V, src, dst)
            assert got_max == ref_max
            assert np.array_equal(got, ref)


def test_noalloc_rejects_edge_count_that_disagrees_with_the_arrays(dc, gpu):
    """The fixed queue ring is sized from E, so E must be the number of
    edges the offset arrays really hold."""
    import torch
    V, src, dst = dc.gen_rmat(10, 8, 24)
    in_off, out_off, out_nbr = _csr(V, src, dst)
    dev = torch.device("cuda", 0)
    t_in = torch.from_numpy(in_off.view(np.int32)).to(dev)
    t_oo = torch.from_numpy(out_off.view(np.int32)).to(dev)
    t_on = torch.from_numpy(np.ascontiguousarray(out_nbr).view(np.int32)).to(dev)
    t_k = torch.zeros(V, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    torch.cuda.synchronize()
    rc = dc.lib().dc_kmax_noalloc(V, len(src) - 1, t_in.data_ptr(), t_oo.data_ptr(), t_on.data_ptr(),
                                  t_k.data_ptr(), None, stream)
    assert rc == -1
    assert "out_off[V]" in dc.last_error()


def test_noalloc_rejects_graphs_beyond_its_limit(dc, gpu):
    rc = dc.lib().dc_kmax_noalloc((1 << 18) + 1, 0, None, None, None, None, None, None)
    assert rc == -5
    assert "limit" in dc.last_error()
