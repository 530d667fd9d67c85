// Seeded synthetic TagMatch workloads (filters with keys, and queries).
//
// The reference ships no benchmark data; its own generator (gen2.cc) uses a
// different hash.  This file fixes one exact, documented definition so that
// every test, the bench and the oracle see byte-identical inputs:
//
//   * RNG: the splitmix64 sequence.  state += 0x9E3779B97F4A7C15, then the
//     splitmix64 finalizer (xor-shift 30 / mul 0xBF58476D1CE4E5B9 / xor-shift
//     27 / mul 0x94D049BB133111EB / xor-shift 31).  Filter draws start from
//     state = fin(seed ^ 0xF1F1F1F1), query draws from fin(seed ^ 0x0E0E0E0E).
//   * Uniform integer in [lo, hi]: lo + ((u64 draw * (hi - lo + 1)) >> 64).
//   * Uniform real in [0, 1): (draw >> 11) * 2^-53.
//   * Zipf(s) over ranks 1..T with P(r) ~ r^-s: inverse CDF by binary search
//     over the cumulative table; the tag id is r - 1.
//   * Tag -> Bloom bits: bit_i(tag) = fin(tag * 256 + i + GOLDEN) mod 192,
//     i = 0..6 (k = 7 hash functions, independent of the workload seed).
//   * A stored filter is the OR of the bits of 1..8 Zipf tags.  Filters are
//     unique: a draw that repeats an existing filter is discarded and drawn
//     again, so every stored filter carries its own 1..4 keys, each uniform in
//     [0, 65536), kept sorted and unique (the per-filter std::set order that
//     tagmatch::add builds, tagmatch.cc:22-77).
//   * A query is, with probability `superset_fraction`, the OR of 1..3
//     uniformly chosen stored filters plus 5..20 extra Zipf tags; otherwise the
//     OR of 10..30 Zipf tags.
//
// Filter and query words use the reference's 32-bit view of a 192-bit filter
// (bitvector.hh:210-212): word w holds bits 32w..32w+31, bit p of the filter
// is bit (p % 32) of word p / 32 -- the little-endian byte image of the
// 24-byte binary record (fib.cc:14-21, test_io.cc:50-68).
#include <cstdint>
#include <cstring>
#include <cmath>
#include <vector>
#include <algorithm>

namespace {

constexpr uint64_t GOLDEN = 0x9E3779B97F4A7C15ull;
constexpr int FILTER_WORDS = 6;
constexpr int FILTER_BITS = 192;
constexpr int HASHES = 7;

inline uint64_t fin64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

struct Rng {
    uint64_t s;
    explicit Rng(uint64_t seed) : s(fin64(seed)) {}
    uint64_t next() { s += GOLDEN; return fin64(s); }
    uint32_t range(uint32_t lo, uint32_t hi) {
        uint64_t span = uint64_t(hi) - lo + 1;
        return lo + uint32_t((static_cast<unsigned __int128>(next()) * span) >> 64);
    }
    uint64_t range64(uint64_t n) {  // uniform in [0, n)
        return uint64_t((static_cast<unsigned __int128>(next()) * n) >> 64);
    }
    double uniform() { return double(next() >> 11) * (1.0 / 9007199254740992.0); }
};

struct Zipf {
    std::vector<double> cdf;
    Zipf(uint32_t n, double s) : cdf(n) {
        double acc = 0.0;
        for (uint32_t r = 1; r <= n; ++r) {
            acc += std::pow(double(r), -s);
            cdf[r - 1] = acc;
        }
        for (auto &c : cdf) c /= acc;
        cdf.back() = 1.0;
    }
    uint32_t draw(Rng &rng) const {
        double u = rng.uniform();
        return uint32_t(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
    }
};

inline void set_tag_bits(uint32_t tag, uint32_t *w) {
    for (int i = 0; i < HASHES; ++i) {
        uint32_t p = uint32_t(fin64(uint64_t(tag) * 256 + uint64_t(i) + GOLDEN) % FILTER_BITS);
        w[p >> 5] |= 1u << (p & 31);
    }
}

inline uint64_t filter_hash(const uint32_t *w) {
    uint64_t h = 0;
    for (int i = 0; i < FILTER_WORDS; ++i) h = fin64(h ^ (uint64_t(w[i]) + GOLDEN * (i + 1)));
    return h;
}

}  // namespace

extern "C" {

// Bit position of hash function i (0..6) for a tag.  Exposed for tests.
uint32_t tmw_tag_bit(uint32_t tag, uint32_t i) {
    return uint32_t(fin64(uint64_t(tag) * 256 + uint64_t(i) + GOLDEN) % FILTER_BITS);
}

// Generates n unique filters.  filters: n*6 words.  key_offsets: n+1 entries.
// keys: capacity 4*n.  Returns the number of keys written, or -1 on bad
// arguments.
int64_t tmw_generate_filters(uint64_t seed, uint64_t n, double zipf_s, uint32_t n_tags,
                             uint32_t *filters, uint32_t *key_offsets, uint32_t *keys) {
    if (n == 0) { key_offsets[0] = 0; return 0; }
    if (!filters || !key_offsets || !keys || n_tags == 0 || n > 0xFFFFFFFFull / 4) return -1;
    Rng rng(seed ^ 0xF1F1F1F1ull);
    Zipf zipf(n_tags, zipf_s);
    // Open-addressing set of filter indices for uniqueness.
    uint64_t cap = 1;
    while (cap < 2 * n) cap <<= 1;
    std::vector<uint32_t> table(cap, 0xFFFFFFFFu);
    uint64_t produced = 0, nkeys = 0;
    uint32_t w[FILTER_WORDS];
    key_offsets[0] = 0;
    uint64_t attempts = 0;
    while (produced < n) {
        if (++attempts > 64 * n + 1000000) return -1;  // tag space exhausted
        std::memset(w, 0, sizeof(w));
        uint32_t ntags = rng.range(1, 8);
        for (uint32_t t = 0; t < ntags; ++t) set_tag_bits(zipf.draw(rng), w);
        uint32_t nk = rng.range(1, 4);
        uint32_t kk[4];
        for (uint32_t k = 0; k < nk; ++k) kk[k] = rng.range(0, 65535);
        uint64_t slot = filter_hash(w) & (cap - 1);
        bool dup = false;
        while (table[slot] != 0xFFFFFFFFu) {
            if (std::memcmp(filters + uint64_t(table[slot]) * FILTER_WORDS, w, sizeof(w)) == 0) { dup = true; break; }
            slot = (slot + 1) & (cap - 1);
        }
        if (dup) continue;
        table[slot] = uint32_t(produced);
        std::memcpy(filters + produced * FILTER_WORDS, w, sizeof(w));
        std::sort(kk, kk + nk);
        uint32_t u = uint32_t(std::unique(kk, kk + nk) - kk);
        for (uint32_t k = 0; k < u; ++k) keys[nkeys++] = kk[k];
        ++produced;
        key_offsets[produced] = uint32_t(nkeys);
    }
    return int64_t(nkeys);
}

// Generates nq queries (nq*6 words) against a stored table of n filters.
int tmw_generate_queries(uint64_t seed, uint64_t nq, const uint32_t *filters, uint64_t n,
                         double zipf_s, uint32_t n_tags, double superset_fraction,
                         uint32_t *queries) {
    if (nq == 0) return 0;
    if (!queries || n_tags == 0 || (superset_fraction > 0.0 && (!filters || n == 0))) return -1;
    Rng rng(seed ^ 0x0E0E0E0Eull);
    Zipf zipf(n_tags, zipf_s);
    for (uint64_t q = 0; q < nq; ++q) {
        uint32_t *w = queries + q * FILTER_WORDS;
        std::memset(w, 0, FILTER_WORDS * sizeof(uint32_t));
        if (rng.uniform() < superset_fraction) {
            uint32_t sets = rng.range(1, 3);
            for (uint32_t s = 0; s < sets; ++s) {
                const uint32_t *f = filters + rng.range64(n) * FILTER_WORDS;
                for (int i = 0; i < FILTER_WORDS; ++i) w[i] |= f[i];
            }
            uint32_t extra = rng.range(5, 20);
            for (uint32_t t = 0; t < extra; ++t) set_tag_bits(zipf.draw(rng), w);
        } else {
            uint32_t tags = rng.range(10, 30);
            for (uint32_t t = 0; t < tags; ++t) set_tag_bits(zipf.draw(rng), w);
        }
    }
    return 0;
}

}  // extern "C"
