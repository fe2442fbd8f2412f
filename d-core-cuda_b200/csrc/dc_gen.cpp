// Seeded synthetic directed graphs: Erdős–Rényi G(n, m) and R-MAT.
//
// The reference ships a non-seedable generator (src/graph_gen.cpp:9-34: unique
// directed edges from std::set and rand() % V, srand(time)).  These generators
// keep its contract -- u != v, no duplicate edges -- and add a seed so that
// every run, test and benchmark sees the same graph.  Both emit the edge list
// sorted by (src, dst), like iterating the reference's std::set.
//
// R-MAT follows Chakrabarti, Zhan & Faloutsos (SDM 2004): each edge picks one
// quadrant per bit with probabilities (a, b, c, d); here the bits are drawn
// MSB first, self-loops are dropped, duplicates are removed by sort-unique and
// vertex labels are optionally permuted by a seeded Fisher-Yates shuffle
// (Graph500 practice) so that degree does not correlate with label.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <unordered_map>
#include <vector>
#include <omp.h>

#include "dc_internal.h"
#include "dc_rng.h"

namespace dc {

// Stable parallel LSD radix sort of 64-bit keys on their low `bits` bits.
void radix_sort_u64(uint64_t* keys, uint64_t* tmp, size_t n, int bits) {
    if (n < 2 || bits <= 0) return;
    const int DIGIT = 16;
    const size_t R = size_t(1) << DIGIT;
    int passes = (bits + DIGIT - 1) / DIGIT;
    int T = std::max(1, std::min(omp_get_max_threads(), int(n / 65536) + 1));
    std::vector<size_t> hist(size_t(T) * R);
    uint64_t* in = keys;
    uint64_t* out = tmp;
    for (int p = 0; p < passes; ++p) {
        int shift = p * DIGIT;
        std::fill(hist.begin(), hist.end(), 0);
#pragma omp parallel num_threads(T)
        {
            int t = omp_get_thread_num();
            size_t lo = n * t / T, hi = n * (t + 1) / T;
            size_t* h = hist.data() + size_t(t) * R;
            for (size_t i = lo; i < hi; ++i) h[(in[i] >> shift) & (R - 1)]++;
#pragma omp barrier
#pragma omp single
            {
                size_t run = 0;
                for (size_t d = 0; d < R; ++d)
                    for (int tt = 0; tt < T; ++tt) {
                        size_t c = hist[size_t(tt) * R + d];
                        hist[size_t(tt) * R + d] = run;
                        run += c;
                    }
            }
            for (size_t i = lo; i < hi; ++i) {
                uint64_t k = in[i];
                out[h[(k >> shift) & (R - 1)]++] = k;
            }
        }
        std::swap(in, out);
    }
    if (in != keys) std::memcpy(keys, in, n * sizeof(uint64_t));
}

}  // namespace dc

using namespace dc;

extern "C" int dc_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t* src, uint32_t* dst) {
    if (n < 2 && m > 0) return dc::set_error(DC_ERR_INVALID, "dc_gen_er: need n >= 2 for m > 0");
    if (m > uint64_t(n) * (n - 1)) return dc::set_error(DC_ERR_INVALID, "dc_gen_er: m exceeds n*(n-1)");
    if (m > 0 && (!src || !dst)) return dc::set_error(DC_ERR_INVALID, "dc_gen_er: null output");
    // open-addressing set of accepted (u, v) keys; key+1 stored so 0 means empty
    size_t cap = 16;
    while (cap < 2 * m + 16) cap <<= 1;
    std::vector<uint64_t> table(cap, 0);
    std::vector<uint64_t> keys;
    keys.reserve(m);
    Xoshiro256ss rng(derive_seed(seed, 0x4552ull));
    while (keys.size() < m) {
        uint32_t u = rng.bounded(n), v = rng.bounded(n);
        if (u == v) continue;
        uint64_t key = (uint64_t(u) << 32) | v;
        uint64_t h = (key * 0x9E3779B97F4A7C15ull) >> 7;
        size_t i = h & (cap - 1);
        bool dup = false;
        while (table[i]) {
            if (table[i] == key + 1) { dup = true; break; }
            i = (i + 1) & (cap - 1);
        }
        if (dup) continue;
        table[i] = key + 1;
        keys.push_back(key);
    }
    std::sort(keys.begin(), keys.end());
    for (uint64_t i = 0; i < m; ++i) {
        src[i] = uint32_t(keys[i] >> 32);
        dst[i] = uint32_t(keys[i]);
    }
    return DC_OK;
}

extern "C" int dc_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                           uint64_t seed, int permute, uint64_t capacity,
                           uint32_t* src, uint32_t* dst, uint64_t* n_edges) {
    if (scale < 1 || scale > 31) return dc::set_error(DC_ERR_INVALID, "dc_gen_rmat: scale must be in [1, 31]");
    if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0))
        return dc::set_error(DC_ERR_INVALID, "dc_gen_rmat: probabilities must be >= 0 with a+b+c <= 1");
    if (!n_edges) return dc::set_error(DC_ERR_INVALID, "dc_gen_rmat: null n_edges");
    const uint64_t V = uint64_t(1) << scale;
    const uint64_t draws = uint64_t(edge_factor) << scale;
    const double two32 = 4294967296.0;
    auto thr = [&](double p) -> uint64_t {
        double t = p * two32;
        if (t >= two32) return uint64_t(1) << 32;
        return uint64_t(t);
    };
    const uint64_t ta = thr(a), tab = thr(a + b), tabc = thr(a + b + c);

    std::vector<uint32_t> perm;
    if (permute) {
        perm.resize(V);
        for (uint64_t i = 0; i < V; ++i) perm[i] = uint32_t(i);
        Xoshiro256ss prng(derive_seed(seed, 0x5045524Dull));
        for (uint64_t i = V - 1; i > 0; --i) {
            uint64_t j = prng.bounded64(i + 1);
            std::swap(perm[i], perm[j]);
        }
    }

    std::vector<uint64_t> keys(draws);
    const uint64_t CHUNK = 1 << 16;
    const uint64_t nchunks = (draws + CHUNK - 1) / CHUNK;
    std::vector<uint64_t> chunk_count(nchunks);
    const uint64_t mask = V - 1;
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t ch = 0; ch < int64_t(nchunks); ++ch) {
        Xoshiro256ss rng(derive_seed(seed, uint64_t(ch)));
        uint64_t lo = uint64_t(ch) * CHUNK, hi = std::min(draws, lo + CHUNK);
        uint64_t w = lo;
        for (uint64_t e = lo; e < hi; ++e) {
            uint64_t u = 0, v = 0;
            uint64_t r64 = 0;
            for (uint32_t lvl = 0; lvl < scale; ++lvl) {
                uint64_t r;
                if ((lvl & 1) == 0) { r64 = rng.next(); r = r64 >> 32; }
                else r = r64 & 0xFFFFFFFFull;
                uint32_t bit = scale - 1 - lvl;
                if (r < ta) {
                } else if (r < tab) {
                    v |= uint64_t(1) << bit;
                } else if (r < tabc) {
                    u |= uint64_t(1) << bit;
                } else {
                    u |= uint64_t(1) << bit;
                    v |= uint64_t(1) << bit;
                }
            }
            if (u == v) continue;
            if (permute) { u = perm[u]; v = perm[v]; }
            keys[w++] = (u << scale) | (v & mask);
        }
        chunk_count[ch] = w - lo;
    }
    // compact chunks (each chunk wrote a prefix of its slot range)
    uint64_t total = 0;
    for (uint64_t ch = 0; ch < nchunks; ++ch) {
        uint64_t lo = ch * CHUNK;
        if (total != lo) std::memmove(keys.data() + total, keys.data() + lo, chunk_count[ch] * sizeof(uint64_t));
        total += chunk_count[ch];
    }
    keys.resize(total);
    {
        std::vector<uint64_t> tmp(total);
        radix_sort_u64(keys.data(), tmp.data(), total, int(2 * scale));
    }
    uint64_t uniq = 0;
    for (uint64_t i = 0; i < total; ++i)
        if (i == 0 || keys[i] != keys[i - 1]) keys[uniq++] = keys[i];
    *n_edges = uniq;
    if (!src || !dst) return DC_OK;  // size query
    if (capacity < uniq) return dc::set_error(DC_ERR_CAPACITY, "dc_gen_rmat: output capacity too small");
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < int64_t(uniq); ++i) {
        src[i] = uint32_t(keys[i] >> scale);
        dst[i] = uint32_t(keys[i] & mask);
    }
    return DC_OK;
}

// Update stream over a graph given as a sorted, duplicate-free edge list:
// n_ops operations, each an insertion of a uniformly random absent edge
// (u != v) with probability insert_frac, otherwise a deletion of a uniformly
// random present edge.  The stream is generated by applying every operation
// to a host copy of the edge set, so it is valid in sequence.
extern "C" int dc_gen_updates(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, uint64_t n_ops,
                              double insert_frac, uint64_t seed, uint32_t* out_u, uint32_t* out_v, uint8_t* out_del) {
    return dc_gen_updates_hot(V, E, src, dst, n_ops, insert_frac, seed, nullptr, 0, nullptr, out_u, out_v, out_del);
}

extern "C" int dc_gen_updates_hot(uint32_t V, uint64_t E, const uint32_t* src, const uint32_t* dst, uint64_t n_ops,
                                  double insert_frac, uint64_t seed, const uint32_t* hot, uint32_t n_hot,
                                  const uint8_t* op_hot, uint32_t* out_u, uint32_t* out_v, uint8_t* out_del) {
    if (V < 2) return dc::set_error(DC_ERR_INVALID, "dc_gen_updates: need V >= 2");
    if (n_ops && (!out_u || !out_v || !out_del)) return dc::set_error(DC_ERR_INVALID, "dc_gen_updates: null output");
    if (op_hot && (!hot || n_hot == 0)) return dc::set_error(DC_ERR_INVALID, "dc_gen_updates_hot: empty hot set");
    std::vector<uint8_t> is_hot;
    if (op_hot) {
        is_hot.assign(V, 0);
        for (uint32_t i = 0; i < n_hot; ++i) {
            if (hot[i] >= V) return dc::set_error(DC_ERR_INVALID, "dc_gen_updates_hot: hot id out of range");
            is_hot[hot[i]] = 1;
        }
    }
    std::vector<uint64_t> keys(E);
    for (uint64_t e = 0; e < E; ++e) {
        if (src[e] >= V || dst[e] >= V) return dc::set_error(DC_ERR_INVALID, "dc_gen_updates: id out of range");
        keys[e] = ((uint64_t)src[e] << 32) | dst[e];
        if (e && keys[e] <= keys[e - 1])
            return dc::set_error(DC_ERR_INVALID, "dc_gen_updates: edges must be sorted by (src, dst) without duplicates");
    }
    std::vector<uint8_t> gone(E, 0);  // original edge deleted
    uint64_t n_gone = 0;
    std::vector<uint64_t> added;      // inserted edges not present originally
    std::unordered_map<uint64_t, uint64_t> added_pos;
    added_pos.reserve(n_ops);
    dc::Xoshiro256ss rng(dc::derive_seed(seed, 0x555044ull));
    // insert when the next 64-bit draw is <= thr (insert_frac of the range);
    // 1.0 and above: always, 0 and below: never (but for an empty graph)
    const uint64_t thr = insert_frac >= 1.0   ? ~0ull
                         : insert_frac <= 0.0 ? 0ull
                                              : (uint64_t)(insert_frac * 18446744073709551616.0);
    auto present = [&](uint64_t k, int64_t* orig) -> bool {
        auto it = std::lower_bound(keys.begin(), keys.end(), k);
        *orig = -1;
        if (it != keys.end() && *it == k) {
            *orig = it - keys.begin();
            return !gone[*orig];
        }
        return added_pos.count(k) != 0;
    };
    for (uint64_t i = 0; i < n_ops; ++i) {
        uint64_t live = E - n_gone + added.size();
        bool ins = rng.next() <= thr || live == 0;
        if (ins && live >= (uint64_t)V * (V - 1)) ins = false;
        // a hot operation has its source among the hot vertices: inserts
        // draw it from them, deletes reject present edges from other sources
        // (up to 4096 draws, then any present edge)
        const bool hot_op = op_hot && op_hot[i];
        if (ins) {
            for (;;) {
                uint32_t u = hot_op ? hot[rng.bounded(n_hot)] : rng.bounded(V), v = rng.bounded(V);
                if (u == v) continue;
                uint64_t k = ((uint64_t)u << 32) | v;
                int64_t orig;
                if (present(k, &orig)) continue;
                if (orig >= 0) {
                    gone[orig] = 0;
                    --n_gone;
                } else {
                    added_pos[k] = added.size();
                    added.push_back(k);
                }
                out_u[i] = u;
                out_v[i] = v;
                out_del[i] = 0;
                break;
            }
        } else {
            for (int tries = 0;; ++tries) {
                uint64_t r = rng.bounded64(E + added.size());
                uint64_t k;
                if (hot_op && tries < 4096) {
                    uint64_t kk = r < E ? keys[r] : added[r - E];
                    if (!is_hot[(uint32_t)(kk >> 32)]) continue;
                }
                if (r < E) {
                    if (gone[r]) continue;
                    gone[r] = 1;
                    ++n_gone;
                    k = keys[r];
                } else {
                    uint64_t j = r - E;
                    k = added[j];
                    uint64_t last = added.back();
                    added[j] = last;
                    added_pos[last] = j;
                    added.pop_back();
                    added_pos.erase(k);
                }
                out_u[i] = (uint32_t)(k >> 32);
                out_v[i] = (uint32_t)k;
                out_del[i] = 1;
                break;
            }
        }
    }
    return DC_OK;
}
