// Insert-batch partition of getKmaxEdgeBatches with KEDGE_BATCHING
// (main.cu:1441-1488), restated in closed form.
//
// The reference gives every edge a root -- the endpoint with the larger kmax,
// the target on ties (main.cu:1449-1452) -- buckets edges by the root's kmax
// in ascending order, and splits each bucket greedily, in input order, into
// sub-batches whose roots are pairwise distinct.  The greedy pass j picks, for
// every root, its j-th remaining edge, so an edge that is the j-th occurrence
// of its root (in input order) lands in pass j of its bucket, and a bucket
// has as many passes as its most frequent root has edges.  One counting pass
// gives the same sub-batch numbering without the per-pass O(V) scans.
#include <algorithm>
#include <cstdint>
#include <unordered_map>
#include <vector>

#include "dc_internal.h"

extern "C" int dc_kmax_edge_batches(uint32_t V, const int32_t* kmaxes, uint64_t B, const uint32_t* from,
                                    const uint32_t* to, int64_t* batch_of, int64_t* n_batches) {
    if (!n_batches || (B && (!kmaxes || !from || !to || !batch_of)))
        return dc::set_error(DC_ERR_INVALID, "dc_kmax_edge_batches: null argument");
    *n_batches = 0;
    if (B == 0) return DC_OK;
    std::vector<int32_t> rk(B);
    std::vector<int64_t> occ(B);
    std::unordered_map<uint32_t, int64_t> seen;
    seen.reserve(B);
    int32_t maxk = 0;
    for (uint64_t e = 0; e < B; ++e) {
        if (from[e] >= V || to[e] >= V) return dc::set_error(DC_ERR_INVALID, "dc_kmax_edge_batches: id out of range");
        uint32_t r = kmaxes[from[e]] > kmaxes[to[e]] ? from[e] : to[e];
        rk[e] = kmaxes[r];
        if (rk[e] < 0) return dc::set_error(DC_ERR_INVALID, "dc_kmax_edge_batches: negative kmax");
        occ[e] = seen[r]++;
        maxk = std::max(maxk, rk[e]);
    }
    std::vector<int64_t> passes((size_t)maxk + 1, 0);
    for (uint64_t e = 0; e < B; ++e) passes[rk[e]] = std::max(passes[rk[e]], occ[e] + 1);
    std::vector<int64_t> base((size_t)maxk + 2, 0);
    for (int32_t k = 0; k <= maxk; ++k) base[k + 1] = base[k] + passes[k];
    for (uint64_t e = 0; e < B; ++e) batch_of[e] = base[rk[e]] + occ[e];
    *n_batches = base[maxk + 1];
    return DC_OK;
}
