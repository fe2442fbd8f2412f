"""Row-cut planner (dc_plan_row_cuts, host only): the cuts it returns reach
the smallest possible largest segment cost, checked against enumeration of
every cut set on staircase and random cumulative cost curves; bad arguments
are rejected."""
import itertools

import numpy as np
import pytest


def _brute(grid, cost, total, ncut):
    best = None
    for comb in itertools.combinations(range(len(grid)), ncut):
        prev, lo = 0.0, 0.0
        for q in comb:
            lo = max(lo, cost[q] - prev)
            prev = cost[q]
        lo = max(lo, total - prev)
        if best is None or lo < best:
            best = lo
    return best


def _longest(grid, cost, total, cuts):
    idx = {g: i for i, g in enumerate(grid)}
    prev, lo = 0.0, 0.0
    for c in cuts:
        lo = max(lo, cost[idx[c]] - prev)
        prev = cost[idx[c]]
    return max(lo, total - prev)


def test_staircase_curve_measured_at_rmat22(dc):
    # cumulative row cost of an R-MAT 22 decomposition at cuts of 5..90 %
    # (ms; few heavy rows make it a staircase), all rows 71.04 ms
    grid = list(range(50, 901, 50))
    cost = [6.03, 11.06, 19.53, 35.13, 35.5, 35.49, 35.37, 41.87, 53.62, 53.62, 53.62, 53.66, 53.64, 53.57,
            54.15, 64.05, 65.67, 65.8]
    total = 71.04
    for ncut in range(1, 8):
        cuts, lo = dc.plan_row_cuts(grid, cost, total, ncut)
        assert cuts == sorted(set(cuts)) and len(cuts) == ncut and all(c in grid for c in cuts)
        assert lo == pytest.approx(_brute(grid, np.float32(cost).tolist(), np.float32(total), ncut), rel=1e-6)
        assert _longest(grid, np.float32(cost).tolist(), np.float32(total), cuts) == pytest.approx(lo, rel=1e-6)
    cuts, lo = dc.plan_row_cuts(grid, cost, total, 3)
    assert lo == pytest.approx(19.53, rel=1e-5)


@pytest.mark.parametrize("seed", range(12))
def test_random_curves_match_enumeration(dc, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 13))
    grid = sorted(rng.choice(np.arange(1, 1000), n, replace=False).tolist())
    steps = rng.exponential(1.0, n + 1) * (rng.random(n + 1) < 0.6)
    cum = np.cumsum(steps).astype(np.float32)
    cost, total = cum[:n].tolist(), float(cum[n])
    if seed % 3 == 0:  # measured curves are noisy: not always monotone
        cost = (np.float32(cost) + rng.normal(0, 0.05, n).astype(np.float32)).tolist()
    for ncut in range(1, min(n, 7) + 1):
        cuts, lo = dc.plan_row_cuts(grid, cost, total, ncut)
        assert cuts == sorted(set(cuts)) and len(cuts) == ncut
        ref = _brute(grid, np.float32(cost).tolist(), np.float32(total), ncut)
        assert lo == pytest.approx(ref, rel=1e-5, abs=1e-6)
        assert _longest(grid, np.float32(cost).tolist(), np.float32(total), cuts) == pytest.approx(lo, rel=1e-5,
                                                                                                     abs=1e-6)


def test_bad_arguments(dc):
    grid, cost = [100, 200, 300], [1.0, 2.0, 3.0]
    for g, c, k in [([100, 100, 300], cost, 1), ([0, 200, 300], cost, 1), ([100, 200, 1000], cost, 1),
                    ([300, 200, 100], cost, 1), (grid, cost, 0), (grid, cost, 4), (grid, cost, 8), ([], [], 1)]:
        with pytest.raises(dc.DCoreError):
            dc.plan_row_cuts(g, c, 4.0, k)
