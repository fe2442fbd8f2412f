/*
 * Seeded graph generators of the CPU oracle -- TEST AND BENCHMARK
 * INFRASTRUCTURE.
 *
 * The benchmark's reference arm times the CPU restatement of the reference's
 * decomposition and must not load the engine library, so it builds its input
 * graphs here.  These functions produce exactly the edge lists of the engine's
 * dc_gen_er / dc_gen_rmat for the same arguments (a CPU test compares them),
 * from the same published algorithms:
 *
 *   splitmix64          Steele, Lea & Flood, "Fast splittable pseudorandom
 *                       number generators" (OOPSLA 2014): seed expansion
 *   xoshiro256**        Blackman & Vigna, "Scrambled linear pseudorandom
 *                       number generators" (TOMS 2021)
 *   bounded integers    Lemire, "Fast random integer generation in an
 *                       interval" (TOMACS 2019), 32-bit multiply-shift with
 *                       rejection; 64-bit ranges by masked rejection
 *   R-MAT               Chakrabarti, Zhan & Faloutsos (SDM 2004): one
 *                       quadrant per bit, most significant bit first
 *   label permutation   Fisher-Yates shuffle (Graph500 practice)
 *
 * The stream layout is the engine's contract for reproducible inputs: a
 * stream seed for (seed, id) is splitmix64 of seed ^ (id * 0xD1342543DE82EF95
 * + 0x2545F4914F6CDD1D); R-MAT draws come in chunks of 65,536 edges, chunk c
 * using stream id c, two 32-bit quadrant draws per 64-bit output (high half
 * first); the permutation uses stream id 0x5045524D, the ER generator stream
 * id 0x4552.  The reference's own generator (src/graph_gen.cpp:9-34) is seeded
 * by time and cannot be reproduced, so it is not restated.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static uint64_t og_splitmix(uint64_t* x) {
    uint64_t z = (*x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

typedef struct { uint64_t s[4]; } og_rng;

static void og_seed(og_rng* r, uint64_t seed) {
    uint64_t x = seed;
    for (int i = 0; i < 4; ++i) r->s[i] = og_splitmix(&x);
}

static uint64_t og_stream(uint64_t seed, uint64_t id) {
    uint64_t x = seed ^ (id * 0xD1342543DE82EF95ull + 0x2545F4914F6CDD1Dull);
    return og_splitmix(&x);
}

static inline uint64_t og_rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }

static inline uint64_t og_next(og_rng* r) {
    uint64_t* s = r->s;
    const uint64_t out = og_rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = og_rotl(s[3], 45);
    return out;
}

/* uniform in [0, n), n >= 1: multiply the top 32 bits by n, reject the
 * low-product values below 2^32 mod n */
static uint32_t og_below32(og_rng* r, uint32_t n) {
    uint64_t m = (og_next(r) >> 32) * (uint64_t)n;
    if ((uint32_t)m < n) {
        const uint32_t reject_below = (uint32_t)(0x100000000ull % n);
        while ((uint32_t)m < reject_below) m = (og_next(r) >> 32) * (uint64_t)n;
    }
    return (uint32_t)(m >> 32);
}

static uint64_t og_below64(og_rng* r, uint64_t n) {
    if (n <= 0xFFFFFFFFull) return og_below32(r, (uint32_t)n);
    uint64_t mask = ~0ull >> __builtin_clzll(n - 1);
    for (;;) {
        uint64_t x = og_next(r) & mask;
        if (x < n) return x;
    }
}

/* LSD radix sort of n keys on their low `bits` bits, 16 bits per pass */
static int og_sort(uint64_t* keys, size_t n, int bits) {
    if (n < 2) return 0;
    uint64_t* tmp = (uint64_t*)malloc(n * sizeof(uint64_t));
    size_t* cnt = (size_t*)malloc(65536 * sizeof(size_t));
    if (!tmp || !cnt) { free(tmp); free(cnt); return -1; }
    uint64_t *in = keys, *out = tmp;
    for (int shift = 0; shift < bits; shift += 16) {
        memset(cnt, 0, 65536 * sizeof(size_t));
        for (size_t i = 0; i < n; ++i) cnt[(in[i] >> shift) & 0xFFFF]++;
        size_t run = 0;
        for (size_t d = 0; d < 65536; ++d) { size_t c = cnt[d]; cnt[d] = run; run += c; }
        for (size_t i = 0; i < n; ++i) out[cnt[(in[i] >> shift) & 0xFFFF]++] = in[i];
        uint64_t* t = in; in = out; out = t;
    }
    if (in != keys) memcpy(keys, in, n * sizeof(uint64_t));
    free(tmp); free(cnt);
    return 0;
}

/*
 * Directed G(n, m): m distinct (u, v), u != v, drawn uniformly (u first, then
 * v), duplicates and self-loops rejected; written sorted by (src, dst).
 * Returns 0, or a negative value on bad arguments / allocation failure.
 */
int og_gen_er(uint32_t n, uint64_t m, uint64_t seed, uint32_t* src, uint32_t* dst) {
    if (m == 0) return 0;
    if (n < 2 || m > (uint64_t)n * (n - 1)) return -1;
    size_t cap = 16;
    while (cap < 2 * m + 16) cap <<= 1;
    uint64_t* seen = (uint64_t*)calloc(cap, sizeof(uint64_t)); /* key + 1, 0 = empty */
    uint64_t* keys = (uint64_t*)malloc(m * sizeof(uint64_t));
    if (!seen || !keys) { free(seen); free(keys); return -3; }
    og_rng r;
    og_seed(&r, og_stream(seed, 0x4552ull));
    uint64_t got = 0;
    while (got < m) {
        uint32_t u = og_below32(&r, n);
        uint32_t v = og_below32(&r, n);
        if (u == v) continue;
        uint64_t key = ((uint64_t)u << 32) | v;
        size_t i = (size_t)((key * 0x9E3779B97F4A7C15ull) >> 7) & (cap - 1);
        int dup = 0;
        while (seen[i]) {
            if (seen[i] == key + 1) { dup = 1; break; }
            i = (i + 1) & (cap - 1);
        }
        if (dup) continue;
        seen[i] = key + 1;
        keys[got++] = key;
    }
    free(seen);
    if (og_sort(keys, m, 64)) { free(keys); return -3; }
    for (uint64_t i = 0; i < m; ++i) {
        src[i] = (uint32_t)(keys[i] >> 32);
        dst[i] = (uint32_t)keys[i];
    }
    free(keys);
    return 0;
}

/*
 * R-MAT with 2^scale vertices and edge_factor * 2^scale draws, quadrant
 * probabilities (a, b, c, 1 - a - b - c) compared against 32-bit draws;
 * self-loops dropped, labels permuted when permute != 0, duplicates removed.
 * Edges sorted by (src, dst).  With src or dst NULL only *n_edges is
 * reported; otherwise capacity must hold them.  Returns 0 or a negative value.
 */
int og_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b, double c, uint64_t seed, int permute,
                uint64_t capacity, uint32_t* src, uint32_t* dst, uint64_t* n_edges) {
    if (scale < 1 || scale > 31 || !n_edges) return -1;
    if (!(a >= 0 && b >= 0 && c >= 0 && a + b + c <= 1.0)) return -1;
    const uint64_t V = 1ull << scale, draws = (uint64_t)edge_factor << scale, mask = V - 1;
    const double two32 = 4294967296.0;
    const double ps[3] = {a, a + b, a + b + c};
    uint64_t th[3];
    for (int i = 0; i < 3; ++i) {
        double t = ps[i] * two32;
        th[i] = t >= two32 ? (1ull << 32) : (uint64_t)t;
    }
    uint32_t* perm = NULL;
    if (permute) {
        perm = (uint32_t*)malloc(V * sizeof(uint32_t));
        if (!perm) return -3;
        for (uint64_t i = 0; i < V; ++i) perm[i] = (uint32_t)i;
        og_rng pr;
        og_seed(&pr, og_stream(seed, 0x5045524Dull));
        for (uint64_t i = V - 1; i > 0; --i) {
            uint64_t j = og_below64(&pr, i + 1);
            uint32_t t = perm[i]; perm[i] = perm[j]; perm[j] = t;
        }
    }
    uint64_t* keys = (uint64_t*)malloc((draws ? draws : 1) * sizeof(uint64_t));
    if (!keys) { free(perm); return -3; }
    /* chunk ch fills a prefix of keys[ch * CHUNK ...]; the prefixes are
     * then packed in chunk order */
    const uint64_t CHUNK = 1ull << 16;
    const int64_t nch = (int64_t)((draws + CHUNK - 1) / CHUNK);
    uint64_t* kept = (uint64_t*)calloc(nch > 0 ? (size_t)nch : 1, sizeof(uint64_t));
    if (!kept) { free(keys); free(perm); return -3; }
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t ch = 0; ch < nch; ++ch) {
        og_rng r;
        og_seed(&r, og_stream(seed, (uint64_t)ch));
        const uint64_t lo = (uint64_t)ch * CHUNK;
        const uint64_t hi = lo + CHUNK < draws ? lo + CHUNK : draws;
        uint64_t n = lo;
        for (uint64_t e = lo; e < hi; ++e) {
            uint64_t u = 0, v = 0, word = 0;
            for (uint32_t lvl = 0; lvl < scale; ++lvl) {
                uint64_t x;
                if (!(lvl & 1)) { word = og_next(&r); x = word >> 32; }
                else x = word & 0xFFFFFFFFull;
                const uint64_t bit = 1ull << (scale - 1 - lvl);
                if (x < th[0]) {
                } else if (x < th[1]) {
                    v |= bit;
                } else if (x < th[2]) {
                    u |= bit;
                } else {
                    u |= bit;
                    v |= bit;
                }
            }
            if (u == v) continue;
            if (perm) { u = perm[u]; v = perm[v]; }
            keys[n++] = (u << scale) | (v & mask);
        }
        kept[ch] = n - lo;
    }
    free(perm);
    uint64_t n = 0;
    for (int64_t ch = 0; ch < nch; ++ch) {
        const uint64_t lo = (uint64_t)ch * CHUNK;
        if (n != lo) memmove(keys + n, keys + lo, kept[ch] * sizeof(uint64_t));
        n += kept[ch];
    }
    free(kept);
    if (og_sort(keys, n, (int)(2 * scale))) { free(keys); return -3; }
    uint64_t uniq = 0;
    for (uint64_t i = 0; i < n; ++i)
        if (i == 0 || keys[i] != keys[i - 1]) keys[uniq++] = keys[i];
    *n_edges = uniq;
    if (src && dst) {
        if (capacity < uniq) { free(keys); return -5; }
        for (uint64_t i = 0; i < uniq; ++i) {
            src[i] = (uint32_t)(keys[i] >> scale);
            dst[i] = (uint32_t)(keys[i] & mask);
        }
    }
    free(keys);
    return 0;
}
