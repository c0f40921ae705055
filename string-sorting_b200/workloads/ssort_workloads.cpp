// ssort_workloads.cpp -- deterministic synthetic string sets for the tests and
// the benchmark (libssort_workloads.so).
//
// The reference measures on text files (one string per line, turned into one
// NUL-separated buffer by sortstring's create_strings_delim,
// src/sortstring.c:310-335).  Its data sets are not available, so these
// generators stand in for them with seeded synthetic inputs of the configured
// shapes.  Every generator writes one arena of NUL-terminated strings plus a
// uint64 offset array (string i starts at arena + offs[i]) and is bitwise
// reproducible for a given seed, independent of the thread count: each chunk of
// CHUNK strings draws from its own stream seeded from (seed, chunk index).
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_set>
#include <vector>
#include <omp.h>

namespace {

constexpr uint64_t CHUNK = 1u << 16;

inline uint64_t splitmix64(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// xoshiro256** (Blackman & Vigna)
struct Rng {
    uint64_t s[4];
    explicit Rng(uint64_t seed) {
        uint64_t x = seed;
        for (auto &w : s) w = splitmix64(x);
    }
    static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    inline uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9;
        const uint64_t t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    // uniform in [0, m)
    inline uint64_t below(uint64_t m) {
        return (uint64_t)(((unsigned __int128)next() * m) >> 64);
    }
    // uniform in [0, 1)
    inline double unit() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

inline uint64_t chunk_seed(uint64_t seed, uint64_t chunk) {
    uint64_t x = seed ^ (chunk * 0xD1B54A32D192ED03ull);
    splitmix64(x);
    return splitmix64(x);
}

// Zipf(s) over ranks 1..N by inverse CDF.
struct Zipf {
    std::vector<double> cdf;
    Zipf(uint64_t N, double s) : cdf(N) {
        double acc = 0;
        for (uint64_t k = 0; k < N; ++k) {
            acc += 1.0 / std::pow((double)(k + 1), s);
            cdf[k] = acc;
        }
        for (auto &c : cdf) c /= acc;
        cdf[N - 1] = 1.0;
    }
    inline uint64_t draw(Rng &r) const {
        double u = r.unit();
        return (uint64_t)(std::upper_bound(cdf.begin(), cdf.end(), u) - cdf.begin());
    }
};

struct Chunked {
    std::vector<std::vector<uint8_t>> text;
    std::vector<std::vector<uint64_t>> local_offs;
};

// Runs gen(rng, out_bytes) for each string (appending the string WITHOUT its
// NUL), chunk-parallel, then concatenates into one malloc'd arena.
template <class F>
int build(uint64_t n, uint64_t seed, F gen, uint8_t **arena_out, uint64_t *bytes_out,
          uint64_t **offs_out) {
    const uint64_t nchunks = (n + CHUNK - 1) / CHUNK;
    Chunked c;
    c.text.resize(nchunks);
    c.local_offs.resize(nchunks);
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t ch = 0; ch < (int64_t)nchunks; ++ch) {
        Rng rng(chunk_seed(seed, (uint64_t)ch));
        const uint64_t lo = (uint64_t)ch * CHUNK;
        const uint64_t hi = std::min(n, lo + CHUNK);
        auto &t = c.text[ch];
        auto &lo_offs = c.local_offs[ch];
        lo_offs.resize(hi - lo);
        t.reserve((hi - lo) * 16);
        for (uint64_t i = lo; i < hi; ++i) {
            lo_offs[i - lo] = t.size();
            gen(rng, t, i);
            t.push_back(0);
        }
    }
    std::vector<uint64_t> base(nchunks + 1, 0);
    for (uint64_t ch = 0; ch < nchunks; ++ch) base[ch + 1] = base[ch] + c.text[ch].size();
    const uint64_t total = base[nchunks];
    // 16 bytes of zero padding after the last string.
    uint8_t *arena = (uint8_t *)std::malloc(total + 16);
    uint64_t *offs = (uint64_t *)std::malloc((n ? n : 1) * sizeof(uint64_t));
    if (!arena || !offs) {
        std::free(arena);
        std::free(offs);
        return -1;
    }
#pragma omp parallel for schedule(dynamic, 1)
    for (int64_t ch = 0; ch < (int64_t)nchunks; ++ch) {
        std::memcpy(arena + base[ch], c.text[ch].data(), c.text[ch].size());
        const uint64_t lo = (uint64_t)ch * CHUNK;
        for (uint64_t k = 0; k < c.local_offs[ch].size(); ++k)
            offs[lo + k] = base[ch] + c.local_offs[ch][k];
        std::vector<uint8_t>().swap(c.text[ch]);
    }
    std::memset(arena + total, 0, 16);
    *arena_out = arena;
    *bytes_out = total;
    *offs_out = offs;
    return 0;
}

}  // namespace

extern "C" {

// Uniform strings: length uniform in [min_len, max_len], each byte uniform over
// alpha_size consecutive values starting at alpha_lo.  With (1, 20, 'a', 26)
// this is the 1,000,000-string plain workload; with the per-instance alphabets
// {4 from 'A', 26 from 'a', 95 from ' '} and length U[1, L] it is the batched
// workload's instance generator.
int ssw_gen_uniform(uint64_t n, uint32_t min_len, uint32_t max_len, uint32_t alpha_lo,
                    uint32_t alpha_size, uint64_t seed, uint8_t **arena, uint64_t *arena_bytes,
                    uint64_t **offs) {
    if (max_len < min_len || alpha_size == 0 || alpha_lo == 0 || alpha_lo + alpha_size > 256)
        return -2;
    const uint64_t span = (uint64_t)max_len - min_len + 1;
    return build(
        n, seed,
        [=](Rng &r, std::vector<uint8_t> &t, uint64_t) {
            const uint64_t len = min_len + r.below(span);
            for (uint64_t k = 0; k < len; ++k) t.push_back((uint8_t)(alpha_lo + r.below(alpha_size)));
        },
        arena, arena_bytes, offs);
}

// Long-shared-prefix URLs: "http://" + one of n_hosts host names (each 8..24
// uniform random lowercase bytes) drawn by Zipf(zipf_s), then 1..6 path
// segments (count uniform), each "/" + 3..12 random [a-z0-9] bytes.
int ssw_gen_urls(uint64_t n, uint32_t n_hosts, double zipf_s, uint64_t seed, uint8_t **arena,
                 uint64_t *arena_bytes, uint64_t **offs) {
    if (n_hosts == 0) return -2;
    std::vector<std::string> hosts(n_hosts);
    {
        Rng r(chunk_seed(seed, 0xFFFFFFFFull));
        for (auto &h : hosts) {
            const uint64_t len = 8 + r.below(17);
            h.resize(len);
            for (auto &ch : h) ch = (char)('a' + r.below(26));
        }
    }
    Zipf z(n_hosts, zipf_s);
    static const char alnum[] = "abcdefghijklmnopqrstuvwxyz0123456789";
    return build(
        n, seed,
        [&](Rng &r, std::vector<uint8_t> &t, uint64_t) {
            static const char pfx[] = "http://";
            t.insert(t.end(), pfx, pfx + 7);
            const std::string &h = hosts[z.draw(r)];
            t.insert(t.end(), h.begin(), h.end());
            const uint64_t segs = 1 + r.below(6);
            for (uint64_t s = 0; s < segs; ++s) {
                t.push_back('/');
                const uint64_t len = 3 + r.below(10);
                for (uint64_t k = 0; k < len; ++k) t.push_back((uint8_t)alnum[r.below(36)]);
            }
        },
        arena, arena_bytes, offs);
}

// Duplicate-heavy words: a vocabulary of vocab distinct words, each of length
// geometric(p_geom) clipped to [1, max_len] with bytes uniform over 'a'..'z';
// every output string is a copy of a vocabulary word drawn by Zipf(zipf_s).
int ssw_gen_zipf_words(uint64_t n, uint32_t vocab, double p_geom, uint32_t max_len,
                       double zipf_s, uint64_t seed, uint8_t **arena, uint64_t *arena_bytes,
                       uint64_t **offs) {
    if (vocab == 0 || max_len == 0 || !(p_geom > 0 && p_geom <= 1)) return -2;
    std::vector<std::string> words;
    words.reserve(vocab);
    {
        std::unordered_set<std::string> seen;
        seen.reserve(vocab * 2);
        Rng r(chunk_seed(seed, 0xFFFFFFFEull));
        uint64_t attempts = 0;
        while (words.size() < vocab) {
            if (++attempts > (uint64_t)vocab * 1000) return -3;
            uint32_t len = 1;
            while (len < max_len && r.unit() >= p_geom) ++len;
            std::string w(len, 'a');
            for (auto &ch : w) ch = (char)('a' + r.below(26));
            if (seen.insert(w).second) words.push_back(std::move(w));
        }
    }
    Zipf z(vocab, zipf_s);
    return build(
        n, seed,
        [&](Rng &r, std::vector<uint8_t> &t, uint64_t) {
            const std::string &w = words[z.draw(r)];
            t.insert(t.end(), w.begin(), w.end());
        },
        arena, arena_bytes, offs);
}

// Independent sort instances in one arena (the batched workload): instance
// k has counts[k] strings of length uniform in [1, max_len[k]] with bytes
// uniform over alpha_size[k] consecutive values from alpha_lo[k].  String
// positions run instance after instance; inst_start (ninst + 1 entries,
// caller-allocated) receives each instance's first position.
int ssw_gen_instances(uint32_t ninst, const uint64_t *counts, const uint32_t *max_len,
                      const uint32_t *alpha_lo, const uint32_t *alpha_size, uint64_t seed,
                      uint32_t *inst_start, uint8_t **arena, uint64_t *arena_bytes,
                      uint64_t **offs) {
    std::vector<uint64_t> start(ninst + 1, 0);
    for (uint32_t k = 0; k < ninst; ++k) {
        if (max_len[k] == 0 || alpha_size[k] == 0 || alpha_lo[k] == 0 ||
            alpha_lo[k] + alpha_size[k] > 256)
            return -2;
        start[k + 1] = start[k] + counts[k];
    }
    const uint64_t n = start[ninst];
    if (n > 0xFFFFFFFEull) return -2;
    for (uint32_t k = 0; k <= ninst; ++k) inst_start[k] = (uint32_t)start[k];
    return build(
        n, seed,
        [&](Rng &r, std::vector<uint8_t> &t, uint64_t i) {
            const uint64_t k =
                (uint64_t)(std::upper_bound(start.begin(), start.end(), i) - start.begin()) - 1;
            const uint64_t len = 1 + r.below(max_len[k]);
            for (uint64_t q = 0; q < len; ++q)
                t.push_back((uint8_t)(alpha_lo[k] + r.below(alpha_size[k])));
        },
        arena, arena_bytes, offs);
}

void ssw_free(void *p) { std::free(p); }

// A deterministic stream of numbers for host-side harnesses (instance sizes,
// arrival times): fills out[0..n) with uniform doubles in [0, 1).
void ssw_uniform_doubles(uint64_t n, uint64_t seed, double *out) {
    Rng r(chunk_seed(seed, 0xFFFFFFFDull));
    for (uint64_t i = 0; i < n; ++i) out[i] = r.unit();
}

int ssw_num_threads(void) { return omp_get_max_threads(); }

}  // extern "C"
