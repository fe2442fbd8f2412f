"""Multi-GPU plumbing around the engine: one process per GPU.

Two ways the path shards (no data-path collective in either):

* rows: every rank holds the whole graph and computes kmax and row 0 itself,
  then a contiguous range of rows 1..kmax chosen from work weights that every
  rank derives identically (dc_row_weights: total degree of C_k); each range
  starts from row 0 restricted to the core of its first row
  (dc_decompose_rows), so ranges are independent.  Rows stay in the HBM of
  the rank that computed them.
* graphs: independent graphs (replicas of the benchmark, serving) are placed
  on ranks by size, largest first onto the least loaded rank.

Timing across ranks is the maximum over ranks of each rank's device time.
"""
import numpy as np


def _pack(w, K, cap):
    """Greedy contiguous packing of rows 1..K under a per-range cost cap."""
    shards, first, acc = [], 1, float(w[1])
    for k in range(2, K + 1):
        if acc + w[k] > cap:
            shards.append((first, k - 1))
            first, acc = k, 2.0 * w[k]  # its first row plus building its counters
        else:
            acc += w[k]
    shards.append((first, K))
    return shards


def row_shards(weights, world):
    """Contiguous ranges [(first, last)] of rows 1..K over `world` ranks, K =
    len(weights) - 1, minimising the largest range cost, where a range costs
    the sum of its rows' weights plus one more weight of its first row for
    starting there (the counters of C_first are built over its members'
    lists; none for the range starting at row 1).  Ranges are
    inclusive and in ascending order; an empty range has first > last."""
    w = np.asarray(weights, np.float64)
    K = len(w) - 1
    if world < 1:
        raise ValueError("world must be >= 1")
    if K < 1:
        return [(1, 0)] * world
    lo, hi = 0.0, float(w[1:].sum()) * 2 + 1.0
    best = _pack(w, K, hi)
    for _ in range(60):
        mid = (lo + hi) / 2
        sh = _pack(w, K, mid)
        if len(sh) <= world:
            best, hi = sh, mid
        else:
            lo = mid
    while len(best) < world:
        best.append((K + 1, K))
    return best


def place_graphs(sizes, world):
    """Rank of every graph: longest-processing-time-first placement."""
    sizes = np.asarray(sizes, np.float64)
    load = np.zeros(world)
    rank = np.zeros(len(sizes), np.int64)
    for i in np.argsort(-sizes, kind="stable"):
        r = int(np.argmin(load))
        rank[i] = r
        load[r] += sizes[i]
    return rank


def max_over_ranks(value, dist=None, device=None):
    """max of a float over the ranks of the default process group (the value
    itself without one)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())
