// Seeded random number generation shared by the graph and update-stream
// generators.  splitmix64 expands a 64-bit seed into generator state and
// xoshiro256** (Blackman & Vigna, "Scrambled linear pseudorandom number
// generators", 2021) produces the stream.  Both are restated from their
// published definitions.
#pragma once
#include <cstdint>

namespace dc {

static inline uint64_t splitmix64_next(uint64_t& x) {
    uint64_t z = (x += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Xoshiro256ss {
    uint64_t s[4];
    explicit Xoshiro256ss(uint64_t seed = 0) { reseed(seed); }
    void reseed(uint64_t seed) {
        uint64_t x = seed;
        for (int i = 0; i < 4; ++i) s[i] = splitmix64_next(x);
    }
    static inline uint64_t rotl(uint64_t v, int k) { return (v << k) | (v >> (64 - k)); }
    inline uint64_t next() {
        const uint64_t result = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return result;
    }
    // Uniform integer in [0, n) without modulo bias (Lemire 2019,
    // "Fast random integer generation in an interval").
    inline uint32_t bounded(uint32_t n) {
        uint64_t m = (next() >> 32) * uint64_t(n);
        uint32_t lo = uint32_t(m);
        if (lo < n) {
            uint32_t t = uint32_t(-n) % n;
            while (lo < t) {
                m = (next() >> 32) * uint64_t(n);
                lo = uint32_t(m);
            }
        }
        return uint32_t(m >> 32);
    }
    inline uint64_t bounded64(uint64_t n) {
        // rejection on the top bits; n > 0
        if (n <= 0xFFFFFFFFull) return bounded(uint32_t(n));
        uint64_t mask = ~0ull;
        uint64_t x = n - 1;
        int lz = __builtin_clzll(x);
        mask >>= lz;
        for (;;) {
            uint64_t r = next() & mask;
            if (r < n) return r;
        }
    }
    // Uniform double in [0, 1) from the top 53 bits.
    inline double uniform() { return double(next() >> 11) * 0x1.0p-53; }
};

// Derives an independent stream seed for (seed, stream id).
static inline uint64_t derive_seed(uint64_t seed, uint64_t stream) {
    uint64_t x = seed ^ (stream * 0xD1342543DE82EF95ull + 0x2545F4914F6CDD1Dull);
    return splitmix64_next(x);
}

}  // namespace dc
