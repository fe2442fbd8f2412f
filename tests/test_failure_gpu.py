"""Failure detection without a GPU fault: every device wait of the engine is
bounded.  A test hook makes one block of the next persistent launch leave
before its first grid barrier, so the barrier that the other blocks wait at
is never completed; their waits run out after the handle's (short) wait
limit, the kernel ends with a status, the call returns DC_ERR_TIMEOUT and
the same handle then decomposes correctly.  Nothing traps, faults or hangs:
the withheld arrival is the flag that nothing sets."""
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("block", [0, 5])
def test_withheld_barrier_arrival_times_out_and_the_handle_recovers(dc, orc, gpu, block):
    V, s, d = dc.gen_rmat(12, 8, 3)
    okm, olm, okmaxes, orows = orc.dcore(V, s, d)
    with dc.Graph.from_edges(V, s, d) as g:
        g.set_wait_limit(200_000_000)  # 200 ms
        g.withhold_barrier(block)
        t0 = time.perf_counter()
        with pytest.raises(dc.DCoreError) as e:
            g.decompose()
        waited = time.perf_counter() - t0
        assert e.value.code == -6, str(e.value)
        assert "wait" in str(e.value)
        assert waited < 3.0  # the handle's limit, not the 4 s default
        # the hook covered one launch: the next call runs to the end
        assert g.decompose() == (okm, olm)
        assert np.array_equal(g.kmaxes(), okmaxes)
        assert np.array_equal(g.rows(), orows)


def test_wait_limit_arguments(dc, gpu):
    V, s, d = dc.gen_rmat(8, 4, 1)
    with dc.Graph.from_edges(V, s, d) as g:
        for bad in (1, 999_999, 600_000_000_001):
            with pytest.raises(dc.DCoreError):
                g.set_wait_limit(bad)
        with pytest.raises(dc.DCoreError):
            g.withhold_barrier(-2)
        g.withhold_barrier(3)
        g.withhold_barrier(-1)  # cancelled before any launch
        g.set_wait_limit(0)
        g.decompose()
