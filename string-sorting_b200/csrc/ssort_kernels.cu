// ssort_kernels.cu -- sm_100a kernels of the MSD radix string sort.
//
// One refinement round works on the live segments at one depth (a multiple of
// 16 bytes).  For every live string it gathers the 16 bytes at arena[off+depth]
// as a big-endian key with every byte after the first NUL zeroed (the
// multi-byte form of the reference's get_char, src/util/get_char.h:42-89, built
// with unsigned shifts; the reference's int-promoted 64-bit form sign-extends
// bytes >= 0x80, :82, and is not reproduced).  Each segment is then sorted by
// (key, index): segments of <= 32 strings by one warp in registers (four
// segments of <= 8 per warp), <= 256 by one warp with up to 8 strings per
// lane, <= SMALL_CAP by a group of 64, 128 or 256 threads of a CTA (by size),
// larger ones are first split by sample partitioning into range buckets and
// equality buckets with a stable scatter.  Equal runs whose key holds no NUL (the reference's
// is_end test, src/util/get_char.h:162-175, and its bucket-skip rule,
// src/msd_ce.cpp:402) become the next round's segments at depth+16; every
// other adjacent pair gets its LCP here.
#include <atomic>

#include "ssort_internal.cuh"

namespace ssort {

namespace {

constexpr uint64_t W_MAX = ~0ull;
constexpr uint32_t IDX_MAX = ~0u;

// ---- 16-byte keys -----------------------------------------------------------
struct Key {
    uint64_t hi, lo;
};

__device__ __forceinline__ Key key_max() { return Key{W_MAX, W_MAX}; }
__device__ __forceinline__ Key to_key(ulonglong2 v) { return Key{v.x, v.y}; }
__device__ __forceinline__ ulonglong2 from_key(Key k) { return make_ulonglong2(k.hi, k.lo); }
__device__ __forceinline__ bool key_lt(const Key &a, const Key &b) {
    return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo);
}
__device__ __forceinline__ bool key_eq(const Key &a, const Key &b) {
    return a.hi == b.hi && a.lo == b.lo;
}
__device__ __forceinline__ bool pair_lt(const Key &a, uint32_t ia, const Key &b, uint32_t ib) {
    return a.hi < b.hi || (a.hi == b.hi && (a.lo < b.lo || (a.lo == b.lo && ia < ib)));
}

__device__ __forceinline__ uint64_t bswap64(uint64_t x) {
    const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    return ((uint64_t)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

// Classic zero-byte test on a little-endian word: the lowest flagged byte is
// the first NUL (no false positives below it).  Returns the word with that
// byte and everything after it cleared, and whether a NUL was found.
__device__ __forceinline__ uint64_t cut_at_nul(uint64_t w, bool &found) {
    const uint64_t z = (w - 0x0101010101010101ull) & ~w & 0x8080808080808080ull;
    found = z != 0;
    if (!found) return w;
    const uint32_t jb = (uint32_t)(__ffsll((long long)z) - 1) >> 3;
    return jb ? (w & ((1ull << (8 * jb)) - 1)) : 0ull;
}

// The 16 bytes of the string at arena[pos..], big-endian, zero after the
// first NUL.  The arena base is 16-byte aligned; bytes at or beyond
// arena_bytes read as NUL.
__device__ __forceinline__ Key load_key(const uint8_t *__restrict__ arena, uint64_t arena_bytes,
                                        uint64_t pos) {
    uint64_t w0, w1;  // little-endian: byte 0 of w0 is arena[pos]
    const uint64_t a = pos & ~15ull;
    const uint32_t off = (uint32_t)(pos & 15);
    // (no a + 32 here: an offset near 2^64 must not wrap into the fast path)
    if (arena_bytes >= 32 && a <= arena_bytes - 32) {
        const ulonglong2 v0 = __ldg(reinterpret_cast<const ulonglong2 *>(arena + a));
        if (off == 0) {
            w0 = v0.x;
            w1 = v0.y;
        } else {
            const ulonglong2 v1 = __ldg(reinterpret_cast<const ulonglong2 *>(arena + a + 16));
            uint64_t q0, q1, q2;
            if (off < 8) {
                q0 = v0.x;
                q1 = v0.y;
                q2 = v1.x;
            } else {
                q0 = v0.y;
                q1 = v1.x;
                q2 = v1.y;
            }
            const uint32_t sh = (off & 7) * 8;
            if (sh) {
                w0 = (q0 >> sh) | (q1 << (64 - sh));
                w1 = (q1 >> sh) | (q2 << (64 - sh));
            } else {
                w0 = q0;
                w1 = q1;
            }
        }
    } else {
        w0 = 0;
        w1 = 0;
        for (int i = 0; i < 16; ++i) {
            const uint64_t q = pos + i;
            if (q >= arena_bytes) break;
            const uint64_t c = arena[q];
            if (i < 8)
                w0 |= c << (8 * i);
            else
                w1 |= c << (8 * (i - 8));
            if (!c) break;
        }
    }
    bool nul;
    w0 = cut_at_nul(w0, nul);
    if (nul)
        w1 = 0;
    else
        w1 = cut_at_nul(w1, nul);
    return Key{bswap64(w0), bswap64(w1)};
}

// The key holds the end of its string (last byte NUL).
__device__ __forceinline__ bool key_is_end(const Key &k) { return (k.lo & 0xFF) == 0; }

__device__ __forceinline__ uint32_t len8(uint64_t w) {
    return w ? 8u - ((uint32_t)(__ffsll((long long)w) - 1) >> 3) : 0u;
}

// Number of string bytes in a key that contains the NUL.
__device__ __forceinline__ uint32_t key_len(const Key &k) {
    return (k.hi & 0xFF) ? 8u + len8(k.lo) : len8(k.hi);
}

// LCP contribution of two keys at the same depth (reference lcp(),
// src/mergesort_lcp.cpp:88-100: stop at the first difference or the NUL).
__device__ __forceinline__ uint32_t key_lcp(const Key &a, const Key &b) {
    if (a.hi != b.hi) return (uint32_t)__clzll((long long)(a.hi ^ b.hi)) >> 3;
    if ((a.hi & 0xFF) == 0) return len8(a.hi);
    if (a.lo != b.lo) return 8u + ((uint32_t)__clzll((long long)(a.lo ^ b.lo)) >> 3);
    return 8u + len8(a.lo);
}

__device__ __forceinline__ uint64_t string_offset(const void *offs, int off_width, uint32_t i) {
    return off_width == 8 ? __ldg(reinterpret_cast<const unsigned long long *>(offs) + i)
                          : (uint64_t)__ldg(reinterpret_cast<const uint32_t *>(offs) + i);
}

__device__ __forceinline__ uint32_t lanemask_lt() {
    uint32_t m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ uint32_t next_pow2(uint32_t x) {
    return x <= 1 ? 1u : 1u << (32 - __clz(x - 1));
}

// Largest i in [0, n) with base[i] <= t (base ascending, base[0] = 0).
__device__ __forceinline__ uint32_t find_seg(const uint32_t *base, uint32_t n, uint32_t t) {
    uint32_t lo = 0, hi = n;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (__ldg(base + mid) <= t)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Lanes of the warp whose value v equals this lane's, for values below
// 2^bits: one ballot per bit (lanes agreeing on every bit are the peers).
// The same set as __match_any_sync(full, v), from vote and logic
// instructions instead of the match unit.  Warp-collective; bits is
// warp-uniform.
__device__ __forceinline__ uint32_t match_bits(uint32_t v, uint32_t bits) {
    uint32_t peers = 0xffffffffu;
    for (uint32_t k = 0; k < bits; ++k) {
        const uint32_t m = __ballot_sync(0xffffffffu, (v >> k) & 1u);
        peers &= ((v >> k) & 1u) ? m : ~m;
    }
    return peers;
}

// Warp-aggregated append to a list counter: all 32 lanes call it together;
// each lane with `want` gets its own slot, at the cost of one atomic per warp
// (appends from millions of small segments would otherwise serialise on one
// address).
// In two steps: warp_reserve issues the warp's atomic without waiting for
// it, so that the reservations a kernel makes on several counters overlap
// their round trips; warp_slot then hands each wanting lane its slot.
struct WarpRes {
    uint32_t mask, base;
};
__device__ __forceinline__ WarpRes warp_reserve(uint32_t *ctr, bool want) {
    const uint32_t mask = __ballot_sync(0xffffffffu, want);
    uint32_t base = 0;
    if (mask && (threadIdx.x & 31) == (uint32_t)(__ffs(mask) - 1))
        base = atomicAdd(ctr, (uint32_t)__popc(mask));
    return WarpRes{mask, base};
}
__device__ __forceinline__ uint32_t warp_slot(const WarpRes &r) {
    if (!r.mask) return 0;  // warp-uniform
    return __shfl_sync(0xffffffffu, r.base, __ffs(r.mask) - 1) + __popc(r.mask & lanemask_lt());
}
__device__ __forceinline__ uint32_t warp_append(uint32_t *ctr, bool want) {
    return warp_slot(warp_reserve(ctr, want));
}

// Append a next-round segment; warp-collective like warp_append.
__device__ __forceinline__ void emit_next_warp(Seg *N, Counters *c, bool want, uint32_t start,
                                               uint32_t len, uint32_t depth) {
    const uint32_t slot = warp_append(&c->n_next, want);
    if (want) N[slot] = Seg{start, len, depth, 0u};
}

// Single-thread append (rare paths only).
__device__ __forceinline__ void emit_next(Seg *N, Counters *c, uint32_t start, uint32_t len,
                                          uint32_t depth) {
    const uint32_t slot = atomicAdd(&c->n_next, 1u);
    N[slot] = Seg{start, len, depth, 0u};
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

// Bucket of `key` among u sorted distinct splitters s[0..u): range bucket 2j
// holds s[j-1] < key < s[j], equality bucket 2j+1 holds key == s[j].  Found
// through the lookup table T: splitters share their first f bits; T[w] counts
// the splitters whose next TBL_BITS bits are below w, so a key strictly
// between the first and last splitter (and hence sharing those f bits) only
// needs a search among the splitters with its own window.
__device__ __forceinline__ uint64_t window64(const Key &k, uint32_t f);

__device__ __forceinline__ uint32_t window_bits(const Key &k, uint32_t f) {
    return (uint32_t)(window64(k, f) >> (64 - TBL_BITS));
}

__device__ __forceinline__ uint32_t classify_tbl(const ulonglong2 *s, const uint16_t *T,
                                                 uint32_t u, uint32_t f, const Key &key) {
    const Key s0 = to_key(s[0]), sl = to_key(s[u - 1]);
    if (key_lt(key, s0)) return 0;
    if (key_eq(key, s0)) return 1;
    if (key_lt(sl, key)) return 2 * u;
    if (key_eq(key, sl)) return 2 * u - 1;
    const uint32_t w = window_bits(key, f);
    uint32_t lo = T[w], hi = T[w + 1];
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (key_lt(to_key(s[mid]), key))
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < u && key_eq(to_key(s[lo]), key)) ? 2 * lo + 1 : 2 * lo;
}

// Asks the memory system to stream the bytes of [p, p + bytes) into L2 (a
// TMA bulk prefetch: no registers, nothing to wait for).  The start is
// rounded up and the end down to 16-byte boundaries, so nothing outside the
// range is touched; ranges are issued in pieces of at most 1 MB.
__device__ __forceinline__ void prefetch_l2(const void *p, uint64_t bytes) {
    uint64_t a = ((uint64_t)(uintptr_t)p + 15) & ~15ull;
    const uint64_t e = ((uint64_t)(uintptr_t)p + bytes) & ~15ull;
    while (a < e) {
        const uint32_t sz = (uint32_t)min(e - a, (uint64_t)(1u << 20));
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(a), "r"(sz) : "memory");
        a += sz;
    }
}

// Padded shared-memory index: one spare slot per 8 keeps both the blocked
// (stride 8) and the striped (stride 1) access patterns free of bank conflicts.
__device__ __forceinline__ uint32_t pad(uint32_t e) { return e + (e >> 3); }

// Slot of record e in a record array: padded (PK, arrays filled by the
// threads themselves) or contiguous (arrays filled by asynchronous copies).
template <bool PK>
__device__ __forceinline__ uint32_t kslot(uint32_t e) {
    if constexpr (PK)
        return pad(e);
    else
        return e;
}

// ---- bitonic sort of (key, index) pairs held in registers -------------------
// Element e = tid * ITEMS + i of a group of THREADS threads (blocked layout).
// Strides below ITEMS run inside a thread, below 32 * ITEMS across lanes with
// shuffles, larger ones through shared memory (groups of several warps).
template <int ITEMS, int J>
__device__ __forceinline__ void stage_local(Key (&k)[ITEMS], uint32_t (&x)[ITEMS], uint32_t kk,
                                            uint32_t tid) {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        if ((i & J) == 0) {
            const int l = i | J;
            const bool asc = (((tid * ITEMS + i) & kk) == 0);
            if (pair_lt(k[l], x[l], k[i], x[i]) == asc) {
                const Key tk = k[i];
                k[i] = k[l];
                k[l] = tk;
                const uint32_t tx = x[i];
                x[i] = x[l];
                x[l] = tx;
            }
        }
    }
}

// Bitonic sort of 32 * ITEMS pairs held by one warp (ITEMS = 2, 4 or 8):
// lane l holds elements l * ITEMS .. l * ITEMS + ITEMS - 1.
template <int ITEMS>
__device__ __forceinline__ void warp_bitonic(Key (&k)[ITEMS], uint32_t (&x)[ITEMS],
                                             uint32_t lane) {
    constexpr uint32_t P = 32 * ITEMS;
#pragma unroll
    for (uint32_t kk = 2; kk <= P; kk <<= 1) {
#pragma unroll
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            if (j >= (uint32_t)ITEMS) {
                const uint32_t lm = j / ITEMS;
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    Key ko;
                    ko.hi = __shfl_xor_sync(0xffffffffu, k[i].hi, lm);
                    ko.lo = __shfl_xor_sync(0xffffffffu, k[i].lo, lm);
                    const uint32_t xo = __shfl_xor_sync(0xffffffffu, x[i], lm);
                    const uint32_t e = lane * ITEMS + i;
                    const bool keep_min = ((lane & lm) == 0) == ((e & kk) == 0);
                    const bool take = keep_min ? pair_lt(ko, xo, k[i], x[i])
                                               : pair_lt(k[i], x[i], ko, xo);
                    if (take) {
                        k[i] = ko;
                        x[i] = xo;
                    }
                }
            } else {
                if constexpr (ITEMS > 4) {
                    if (j == 4) {
                        stage_local<ITEMS, 4>(k, x, kk, lane);
                        continue;
                    }
                }
                if constexpr (ITEMS > 2) {
                    if (j == 2) {
                        stage_local<ITEMS, 2>(k, x, kk, lane);
                        continue;
                    }
                }
                if constexpr (ITEMS > 1) stage_local<ITEMS, 1>(k, x, kk, lane);
            }
        }
    }
}

// One warp sorts the 32 * ITEMS pairs at padded shared-memory positions
// base .. base + 32 * ITEMS - 1 in place.
template <int ITEMS, bool PK = true>
__device__ __noinline__ void warp_sort_run(ulonglong2 *sk, uint32_t *sx, uint32_t base,
                                              uint32_t lane) {
    Key k[ITEMS];
    uint32_t x[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint32_t e = base + lane * ITEMS + i;
        k[i] = to_key(sk[kslot<PK>(e)]);
        x[i] = sx[kslot<PK>(e)];
    }
    warp_bitonic<ITEMS>(k, x, lane);
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint32_t e = base + lane * ITEMS + i;
        sk[kslot<PK>(e)] = from_key(k[i]);
        sx[kslot<PK>(e)] = x[i];
    }
}

// ---- packed 64-bit sort keys -------------------------------------------------
// Within one segment every key shares its first f bits (f = leading zeros of
// the OR of key ^ key0 over the segment).  The 53 bits after them, with the
// string's local position (< 2048) in the low 11 bits, form a unique 64-bit
// sort key whose order agrees with (key, index) order except between keys
// whose windows are equal; those pairs are checked afterwards (check_sorted)
// and a segment with any disagreement is re-sorted with the full comparator.
constexpr uint32_t POS_BITS = 11;
constexpr uint64_t POS_MASK = (1ull << POS_BITS) - 1;

__device__ __forceinline__ uint32_t clz128(uint64_t hi, uint64_t lo) {
    return hi ? (uint32_t)__clzll((long long)hi)
              : 64u + (lo ? (uint32_t)__clzll((long long)lo) : 64u);
}

// Top 64 bits of the 128-bit key shifted left by f (0 <= f < 128).
__device__ __forceinline__ uint64_t window64(const Key &k, uint32_t f) {
    if (f == 0) return k.hi;
    if (f < 64) return (k.hi << f) | (k.lo >> (64 - f));
    return k.lo << (f - 64);
}

__device__ __forceinline__ uint64_t sort_key(const Key &k, uint32_t f, uint32_t pos) {
    return (window64(k, f) & ~POS_MASK) | pos;
}

template <int ITEMS, int J, typename V = uint64_t>
__device__ __forceinline__ void stage_local64(V (&v)[ITEMS], uint32_t kk, uint32_t lane) {
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        if ((i & J) == 0) {
            const int l = i | J;
            const bool asc = (((lane * ITEMS + i) & kk) == 0);
            const V a = v[i], b = v[l];
            const bool sw = (b < a) == asc;
            v[i] = sw ? b : a;
            v[l] = sw ? a : b;
        }
    }
}

// Bitonic sort of 32 * ITEMS distinct uint64 values held by one warp (lane l
// holds elements l * ITEMS ..), ITEMS = 1, 2, 4 or 8.
template <int ITEMS, typename V = uint64_t>
__device__ __forceinline__ void warp_bitonic64(V (&v)[ITEMS], uint32_t lane) {
    constexpr uint32_t P = 32 * ITEMS;
#pragma unroll
    for (uint32_t kk = 2; kk <= P; kk <<= 1) {
#pragma unroll
        for (uint32_t j = kk >> 1; j > 0; j >>= 1) {
            if (j >= (uint32_t)ITEMS) {
                const uint32_t lm = j / ITEMS;
#pragma unroll
                for (int i = 0; i < ITEMS; ++i) {
                    const V o = __shfl_xor_sync(0xffffffffu, v[i], lm);
                    const uint32_t e = lane * ITEMS + i;
                    const bool keep_min = ((lane & lm) == 0) == ((e & kk) == 0);
                    v[i] = keep_min ? (o < v[i] ? o : v[i]) : (o > v[i] ? o : v[i]);
                }
            } else {
                if constexpr (ITEMS > 4) {
                    if (j == 4) {
                        stage_local64<ITEMS, 4, V>(v, kk, lane);
                        continue;
                    }
                }
                if constexpr (ITEMS > 2) {
                    if (j == 2) {
                        stage_local64<ITEMS, 2, V>(v, kk, lane);
                        continue;
                    }
                }
                if constexpr (ITEMS > 1) stage_local64<ITEMS, 1, V>(v, kk, lane);
            }
        }
    }
}

// Merge-path split over two sorted uint64 runs (values distinct).
template <typename V = uint64_t>
__device__ __forceinline__ uint32_t merge_split64(const V *s, uint32_t a0, uint32_t la,
                                                  uint32_t b0, uint32_t lb, uint32_t d) {
    uint32_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (s[pad(a0 + mid)] < s[pad(b0 + d - 1 - mid)])
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// Merge-path split: number of elements of run A (length la, at a0) among the
// first d outputs of merging A with run B (length lb, at b0); ties go to A.
template <bool PK = true>
__device__ __forceinline__ uint32_t merge_split(const ulonglong2 *sk, const uint32_t *sx,
                                                uint32_t a0, uint32_t la, uint32_t b0,
                                                uint32_t lb, uint32_t d) {
    uint32_t lo = d > lb ? d - lb : 0, hi = d < la ? d : la;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        const uint32_t pa = kslot<PK>(a0 + mid), pb = kslot<PK>(b0 + d - 1 - mid);
        // A[mid] <= B[d-1-mid]: A[mid] is among the first d outputs.
        if (!pair_lt(to_key(sk[pb]), sx[pb], to_key(sk[pa]), sx[pa]))
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// After a segment of `len` strings is sorted into shared memory (padded
// layout), write its indices, LCPs and first/last keys, and emit the runs of
// equal non-final keys as next-round segments.  Called by `threads` threads
// numbered t = 0..threads-1.
// Sorted position e -> shared-memory slot of its record: the slot itself
// (records already in order) or the position field of the e-th packed key.
template <bool IND, bool PK = true>
__device__ __forceinline__ uint32_t rec_slot(const uint64_t *sv, uint32_t e) {
    if constexpr (IND)
        return kslot<PK>((uint32_t)(sv[pad(e)] & POS_MASK));
    else
        return kslot<PK>(e);
}

template <bool IND, bool PK = true>
__device__ __forceinline__ void finish_segment(const SortArgs &a, const Seg &s,
                                               const ulonglong2 *sk, const uint32_t *sx,
                                               const uint64_t *sv, uint32_t t, uint32_t threads,
                                               Seg *N, Counters *c) {
    // Uniform trip count so that every warp reaches the collective append.
    for (uint32_t e0 = 0; e0 < s.len; e0 += threads) {
        const uint32_t e = e0 + t;
        bool want = false;
        uint32_t run_lo = 0;
        if (e < s.len) {
            const uint32_t p = s.start + e;
            const uint32_t q = rec_slot<IND, PK>(sv, e);
            const Key k = to_key(sk[q]);
            a.idx[0][p] = sx[q];
            if (e == 0 || e == s.len - 1) a.key[0][p] = from_key(k);
            bool same_prev = false;
            if (e > 0) {
                const Key kp = to_key(sk[rec_slot<IND, PK>(sv, e - 1)]);
                same_prev = key_eq(kp, k);
                if (!same_prev)
                    a.lcp[p] = s.depth + key_lcp(kp, k);
                else if (key_is_end(k))
                    a.lcp[p] = s.depth + key_len(k);
            }
            if (same_prev && !key_is_end(k) &&
                (e == s.len - 1 || !key_eq(to_key(sk[rec_slot<IND, PK>(sv, e + 1)]), k))) {
                uint32_t lo = 0, hi = e;  // first position of this run
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (key_lt(to_key(sk[rec_slot<IND, PK>(sv, mid)]), k))
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                want = true;
                run_lo = lo;
            }
        }
        emit_next_warp(N, c, want, s.start + run_lo, e - run_lo + 1, s.depth + KEY_BYTES);
    }
}

// finish_segment for a packed sort whose order lives in sv (records in place):
// neighbours whose windows differ get their LCP from the windows alone (all
// keys share their first f bits, so the first differing bit is f + the
// leading zeros of the windows' xor, and no NUL can precede it in either
// key); only neighbours with equal windows read their full keys.  Same
// writes and next-round runs as finish_segment<true>.
template <bool PK>
__device__ __forceinline__ void finish_packed(const SortArgs &a, const Seg &s,
                                              const ulonglong2 *sk, const uint32_t *sx,
                                              const uint64_t *sv, uint32_t f, uint32_t t,
                                              uint32_t threads, Seg *N, Counters *c) {
    // Uniform trip count so that every warp reaches the collective append.
    for (uint32_t e0 = 0; e0 < s.len; e0 += threads) {
        const uint32_t e = e0 + t;
        bool want = false;
        uint32_t run_lo = 0;
        if (e < s.len) {
            const uint32_t p = s.start + e;
            const uint64_t v = sv[pad(e)];
            const uint32_t q = kslot<PK>((uint32_t)(v & POS_MASK));
            a.idx[0][p] = sx[q];
            if (e == 0 || e == s.len - 1) a.key[0][p] = sk[q];
            bool same_prev = false;
            Key k = key_max();
            if (e > 0) {
                const uint64_t vp = sv[pad(e - 1)];
                const uint64_t x = (v ^ vp) & ~POS_MASK;
                if (x) {
                    a.lcp[p] = s.depth + ((f + (uint32_t)__clzll((long long)x)) >> 3);
                } else {
                    k = to_key(sk[q]);
                    const Key kp = to_key(sk[kslot<PK>((uint32_t)(vp & POS_MASK))]);
                    same_prev = key_eq(kp, k);
                    if (!same_prev)
                        a.lcp[p] = s.depth + key_lcp(kp, k);
                    else if (key_is_end(k))
                        a.lcp[p] = s.depth + key_len(k);
                }
            }
            if (same_prev && !key_is_end(k)) {
                // a run of equal keys that do not end: is this its last record?
                bool last = e == s.len - 1;
                if (!last) {
                    const uint64_t vn = sv[pad(e + 1)];
                    last = ((v ^ vn) & ~POS_MASK) != 0 ||
                           !key_eq(to_key(sk[kslot<PK>((uint32_t)(vn & POS_MASK))]), k);
                }
                if (last) {
                    uint32_t lo = 0, hi = e;  // first position of this run
                    while (lo < hi) {
                        const uint32_t mid = (lo + hi) >> 1;
                        const uint32_t qm = kslot<PK>((uint32_t)(sv[pad(mid)] & POS_MASK));
                        if (key_lt(to_key(sk[qm]), k))
                            lo = mid + 1;
                        else
                            hi = mid;
                    }
                    want = true;
                    run_lo = lo;
                }
            }
        }
        emit_next_warp(N, c, want, s.start + run_lo, e - run_lo + 1, s.depth + KEY_BYTES);
    }
}

// True when the sorted order (through the packed keys) agrees with full
// (key, index) order wherever the packed keys could not tell records apart
// (equal windows).  Called by `threads` threads numbered t; per-thread verdict.
template <bool PK = true>
__device__ __forceinline__ bool window_pairs_ok_ind(const ulonglong2 *sk, const uint64_t *sv,
                                                    uint32_t len, uint32_t t, uint32_t threads) {
    bool ok = true;
    for (uint32_t e = t + 1; e < len; e += threads) {
        const uint64_t va = sv[pad(e - 1)], vb = sv[pad(e)];
        if ((va >> POS_BITS) == (vb >> POS_BITS)) {
            const Key kp = to_key(sk[kslot<PK>((uint32_t)(va & POS_MASK))]);
            const Key k = to_key(sk[kslot<PK>((uint32_t)(vb & POS_MASK))]);
            if (key_lt(k, kp)) ok = false;
        }
    }
    return ok;
}

// Runs of equal windows after a packed sort hold their records in position
// order.  window_runs_short: no run is longer than FIX_RUN_CAP (else the
// caller sorts the whole segment with the full comparator).  sort_window_runs:
// the thread that owns a run's first element puts the run into full (key,
// position) order in place (insertion sort: equal keys keep position order).
// Runs are disjoint and every entry of a run has the run's window bits, so
// the neighbours another thread reads keep their windows while it sorts.
constexpr uint32_t FIX_RUN_CAP = 64;

__device__ __forceinline__ bool window_run_start(const uint64_t *sv, uint32_t len, uint32_t e) {
    const uint64_t w = sv[pad(e)] >> POS_BITS;
    return e + 1 < len && (sv[pad(e + 1)] >> POS_BITS) == w &&
           (e == 0 || (sv[pad(e - 1)] >> POS_BITS) != w);
}

__device__ __forceinline__ bool window_runs_short(const uint64_t *sv, uint32_t len, uint32_t t,
                                                  uint32_t threads) {
    for (uint32_t e = t; e + 1 < len; e += threads) {
        if (!window_run_start(sv, len, e)) continue;
        const uint64_t w = sv[pad(e)] >> POS_BITS;
        const uint32_t r = min(len, e + FIX_RUN_CAP + 1);
        uint32_t q = e + 2;
        while (q < r && (sv[pad(q)] >> POS_BITS) == w) ++q;
        if (q - e > FIX_RUN_CAP) return false;
    }
    return true;
}

template <bool PK = true>
__device__ __forceinline__ void sort_window_runs(const ulonglong2 *sk, uint64_t *sv, uint32_t len,
                                                 uint32_t t, uint32_t threads) {
    for (uint32_t e = t; e + 1 < len; e += threads) {
        if (!window_run_start(sv, len, e)) continue;
        const uint64_t w = sv[pad(e)] >> POS_BITS;
        uint32_t r = e + 2;
        while (r < len && (sv[pad(r)] >> POS_BITS) == w) ++r;
        for (uint32_t i = e + 1; i < r; ++i) {
            const uint64_t v = sv[pad(i)];
            const Key kv = to_key(sk[kslot<PK>((uint32_t)(v & POS_MASK))]);
            uint32_t j = i;
            while (j > e) {
                const uint64_t u = sv[pad(j - 1)];
                if (!key_lt(kv, to_key(sk[kslot<PK>((uint32_t)(u & POS_MASK))]))) break;
                sv[pad(j)] = u;
                --j;
            }
            sv[pad(j)] = v;
        }
    }
}

// 32-bit packed keys for a first sort: the 21 window bits after the common
// prefix and the 11-bit position.  Their order is the 64-bit packed order
// except among keys whose 21 bits tie; see block_class.
constexpr uint32_t NARROW_SHIFT = 64 - 21;  // 64-bit packed key >> this = the 21 bits

__device__ __forceinline__ uint32_t sort_key32(const Key &k, uint32_t f, uint32_t pos) {
    return (uint32_t)(window64(k, f) >> 32) & ~(uint32_t)POS_MASK | pos;
}

// In sv[0..len), the 64-bit packed keys of records in 32-bit order: runs of
// keys whose top 21 bits tie are put into 64-bit order in place by the
// thread that owns the run's first entry (insertion sort); returns false in
// that thread when a run is longer than FIX_RUN_CAP (the caller then sorts
// the segment on 64-bit keys from scratch).
__device__ __forceinline__ bool sort_narrow_runs(uint64_t *sv, uint32_t len, uint32_t t,
                                                 uint32_t threads) {
    bool ok = true;
    for (uint32_t e = t; e + 1 < len; e += threads) {
        const uint64_t w = sv[pad(e)] >> NARROW_SHIFT;
        if ((sv[pad(e + 1)] >> NARROW_SHIFT) != w) continue;
        if (e > 0 && (sv[pad(e - 1)] >> NARROW_SHIFT) == w) continue;  // not the run's start
        uint32_t r = e + 2;
        while (r < len && (sv[pad(r)] >> NARROW_SHIFT) == w && r - e <= FIX_RUN_CAP) ++r;
        if (r - e > FIX_RUN_CAP) {
            ok = false;
            continue;
        }
        for (uint32_t i = e + 1; i < r; ++i) {
            const uint64_t v = sv[pad(i)];
            uint32_t j = i;
            while (j > e && sv[pad(j - 1)] > v) {
                sv[pad(j)] = sv[pad(j - 1)];
                --j;
            }
            sv[pad(j)] = v;
        }
    }
    return ok;
}

template <int ITEMS>
__device__ __forceinline__ void warp_run_packed32(const ulonglong2 *sk, uint32_t *sv32,
                                                  uint32_t base, uint32_t len, uint32_t f,
                                                  uint32_t lane) {
    uint32_t v[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint32_t e = base + lane * ITEMS + i;
        v[i] = e < len ? sort_key32(to_key(sk[pad(e)]), f, e) : ~0u;
    }
    warp_bitonic64<ITEMS, uint32_t>(v, lane);
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) sv32[pad(base + lane * ITEMS + i)] = v[i];
}

// Compare-exchange: afterwards a <= b.
__device__ __forceinline__ void cas64(uint64_t &a, uint64_t &b) {
    const bool lt = a < b;
    const uint64_t lo = lt ? a : b, hi = lt ? b : a;
    a = lo;
    b = hi;
}

// Sorts ITEMS (2, 4 or 8) values held by one thread: optimal sorting networks
// of 1, 5 and 19 comparators.
template <int ITEMS>
__device__ __forceinline__ void sort_local64(uint64_t (&v)[ITEMS]) {
    if constexpr (ITEMS == 2) {
        cas64(v[0], v[1]);
    } else if constexpr (ITEMS == 4) {
        cas64(v[0], v[1]); cas64(v[2], v[3]);
        cas64(v[0], v[2]); cas64(v[1], v[3]);
        cas64(v[1], v[2]);
    } else {
        static_assert(ITEMS == 8, "2, 4 or 8 values per thread");
        cas64(v[0], v[2]); cas64(v[1], v[3]); cas64(v[4], v[6]); cas64(v[5], v[7]);
        cas64(v[0], v[4]); cas64(v[1], v[5]); cas64(v[2], v[6]); cas64(v[3], v[7]);
        cas64(v[0], v[1]); cas64(v[2], v[3]); cas64(v[4], v[5]); cas64(v[6], v[7]);
        cas64(v[2], v[4]); cas64(v[3], v[5]);
        cas64(v[1], v[4]); cas64(v[3], v[6]);
        cas64(v[1], v[2]); cas64(v[3], v[4]); cas64(v[5], v[6]);
    }
}

// One warp sorts the 32 * ITEMS values v (lane l holds any ITEMS of them)
// into sv[pad(base .. base + 32 * ITEMS)]: every lane sorts its own values in
// registers, then merge-path passes (synchronised by __syncwarp only) double
// the sorted runs up to the whole warp.  Fewer instructions than the bitonic
// network, whose 15 cross-lane stages each move every value through a
// shuffle; equal values (the all-ones padding) merge consistently.
template <int ITEMS>
__device__ __forceinline__ void warp_merge_sort64(uint64_t (&v)[ITEMS], uint64_t *sv,
                                                  uint32_t base, uint32_t lane) {
    sort_local64<ITEMS>(v);
    const uint32_t o = lane * ITEMS;
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) sv[pad(base + o + i)] = v[i];
    __syncwarp();
#pragma unroll
    for (uint32_t run = ITEMS; run < 32 * ITEMS; run <<= 1) {
        const uint32_t a0 = base + (o & ~(2 * run - 1)), b0 = a0 + run;
        const uint32_t d = o & (2 * run - 1);
        uint32_t ia = merge_split64(sv, a0, run, b0, run, d);
        uint32_t ib = d - ia;
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) {
            const uint64_t va = ia < run ? sv[pad(a0 + ia)] : ~0ull;
            const uint64_t vb = ib < run ? sv[pad(b0 + ib)] : ~0ull;
            const bool take_a = ib >= run || (ia < run && va < vb);
            v[i] = take_a ? va : vb;
            ia += take_a;
            ib += !take_a;
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) sv[pad(base + o + i)] = v[i];
        __syncwarp();
    }
}

// One warp: packed keys of the records at slots base .. base + 32*ITEMS - 1
// (positions >= len pad with all-ones), sorted, stored to sv; by the bitonic
// network or (MERGE) by warp_merge_sort64.
template <int ITEMS, bool MERGE = false>
__device__ __forceinline__ void warp_run_packed(const ulonglong2 *sk, uint64_t *sv,
                                                uint32_t base, uint32_t len, uint32_t f,
                                                uint32_t lane) {
    uint64_t v[ITEMS];
#pragma unroll
    for (int i = 0; i < ITEMS; ++i) {
        const uint32_t e = base + lane * ITEMS + i;
        v[i] = e < len ? sort_key(to_key(sk[pad(e)]), f, e) : ~0ull;
    }
    if constexpr (MERGE) {
        warp_merge_sort64<ITEMS>(v, sv, base, lane);
    } else {
        warp_bitonic64<ITEMS>(v, lane);
#pragma unroll
        for (int i = 0; i < ITEMS; ++i) sv[pad(base + lane * ITEMS + i)] = v[i];
    }
}

// ---------------------------------------------------------------------------
__global__ void k_iota(uint32_t *idx, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        idx[i] = i;
}

// Appends o (when sm) to the CTA-sort list of its size class; warp-collective.
// Appends segment o (when v) to the list its length selects: one-warp sorts
// of <= 32 or <= warp8_cap strings, the CTA sorts' three size classes, or the
// large list L (counter nl).  Warp-collective; the six reservations are all
// issued before any is waited for.
__device__ __forceinline__ void append_by_length(const Seg &o, bool v, uint32_t warp8_cap,
                                                 Seg *W1, Seg *W8, const SmallLists &S, Seg *L,
                                                 uint32_t *nl, Counters *c) {
    const bool w1 = v && o.len <= (uint32_t)WARP1_CAP;
    const bool w8 = v && !w1 && o.len <= warp8_cap;
    const bool sm = v && !w1 && !w8 && o.len <= (uint32_t)SMALL_CAP;
    const bool c0 = sm && o.len <= (uint32_t)BLOCK_CAP1;
    const bool c1 = sm && !c0 && o.len <= (uint32_t)BLOCK_CAP2;
    const bool c2 = sm && !c0 && !c1;
    const bool lg = v && !w1 && !w8 && !sm;
    const WarpRes r1 = warp_reserve(&c->n_w1, w1), r8 = warp_reserve(&c->n_w8, w8),
                  rs0 = warp_reserve(&c->n_small, c0), rs1 = warp_reserve(&c->n_small2, c1),
                  rs2 = warp_reserve(&c->n_small3, c2), rl = warp_reserve(nl, lg);
    const uint32_t t1 = warp_slot(r1), t8 = warp_slot(r8), ts0 = warp_slot(rs0),
                   ts1 = warp_slot(rs1), ts2 = warp_slot(rs2), tl = warp_slot(rl);
    if (w1) W1[t1] = o;
    if (w8) W8[t8] = o;
    if (c0) S.s[0][ts0] = o;
    if (c1) S.s[1][ts1] = o;
    if (c2) S.s[2][ts2] = o;
    if (lg) L[tl] = o;
}

__global__ void k_classify(const Seg *__restrict__ R, Count cnt, uint32_t warp8_cap, Seg *W1,
                           Seg *W8, SmallLists S, Seg *L, Counters *c) {
    const uint32_t nR = count_of(cnt);
    // Block-uniform trip count: every warp reaches the collective appends.
    for (uint32_t b0 = blockIdx.x * blockDim.x; b0 < nR; b0 += gridDim.x * blockDim.x) {
    const uint32_t i = b0 + threadIdx.x;
    const bool v = i < nR;
    const Seg s = v ? R[i] : Seg{0, 0, 0, 0};
    append_by_length(s, v, warp8_cap, W1, W8, S, L, &c->n_large, c);
    const bool lg = v && s.len > (uint32_t)SMALL_CAP && s.len > warp8_cap;
    const unsigned long long live = warp_sum(v ? s.len : 0);
    const unsigned long long big = warp_sum(lg ? s.len : 0);
    if ((threadIdx.x & 31) == 0) {
        if (live) atomicAdd(&c->live_next, live);
        if (big) atomicAdd(&c->gather_elems, big);
    }
    }
}

// ---- batches of independent instances ---------------------------------------
// Instance i owns positions inst_start[i] .. inst_start[i+1]-1: it enters
// round 0 as its own segment, and its first LCP entry is 0.
__global__ void k_init_batch(const uint32_t *__restrict__ inst_start, uint32_t ninst, Seg *R,
                             uint32_t *lcp, Counters *c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool v = i < ninst;
    const uint32_t s = v ? inst_start[i] : 0, e = v ? inst_start[i + 1] : 0;
    if (v && e > s) lcp[s] = 0;
    const bool seg = v && e - s >= 2;
    const uint32_t slot = warp_append(&c->n_next, seg);
    if (seg) R[slot] = Seg{s, e - s, 0, 0};
}

// Global positions -> indices within each position's instance.
__global__ void k_localize(uint32_t *perm, uint32_t n, const uint32_t *__restrict__ inst_start,
                           uint32_t ninst) {
    for (uint32_t p = blockIdx.x * blockDim.x + threadIdx.x; p < n; p += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = ninst;  // largest i with inst_start[i] <= p
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(inst_start + mid) <= p)
                lo = mid;
            else
                hi = mid;
        }
        perm[p] -= __ldg(inst_start + lo);
    }
}

// ---- request server: joining and retiring requests between rounds ----------
// The requests of one step are described by ReqJob records; a flat index q
// over all their positions (jobs[j].first = positions of the jobs before j)
// finds its job by binary search.
__device__ __forceinline__ uint32_t find_job(const ReqJob *__restrict__ jobs, uint32_t njobs,
                                             uint32_t q) {
    uint32_t lo = 0, hi = njobs;  // largest j with jobs[j].first <= q
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (jobs[mid].first <= q)
            lo = mid;
        else
            hi = mid;
    }
    return lo;
}

// Joins admitted requests: request j occupies positions [pos, pos + n) and its
// bytes sit at region_base in the pool arena.  Its offsets arrive either as
// uint64 in place in goffs or as uint32 staged in lcp at its positions; each
// becomes a pool offset.  An offset at or past the request's own arena_bytes
// is clamped to arena_bytes, where the server stores a NUL byte: the same
// empty string the single-request sort reads past the end of its arena.
// Positions get their identity index, lcp of the first position becomes 0,
// and a request of two or more strings becomes one depth-0 segment at
// R[slot].
__global__ void k_join(uint64_t *goffs, uint32_t *lcp, uint32_t *perm,
                       const ReqJob *__restrict__ jobs, uint32_t njobs, uint32_t total, Seg *R) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += gridDim.x * blockDim.x) {
        const ReqJob jb = jobs[find_job(jobs, njobs, q)];
        const uint32_t i = q - jb.first;
        const uint32_t p = jb.pos + i;
        uint64_t o = jb.off_width == 4 ? (uint64_t)lcp[p] : goffs[p];
        if (o > jb.arena_bytes) o = jb.arena_bytes;
        goffs[p] = jb.region_base + o;
        perm[p] = p;
        if (i == 0) {
            lcp[p] = 0;
            if (jb.n >= 2) R[jb.slot] = Seg{jb.pos, jb.n, 0, 0};
        }
    }
}

// flag[j] = 1 for every active request j that still owns a segment of R;
// base[] holds the active requests' first positions in ascending order.
__global__ void k_mark(const Seg *__restrict__ R, uint32_t nR, const uint32_t *__restrict__ base,
                       uint32_t nact, uint32_t *flag) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nR;
         i += gridDim.x * blockDim.x) {
        const uint32_t s = R[i].start;
        uint32_t lo = 0, hi = nact;  // largest j with base[j] <= s
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (__ldg(base + mid) <= s)
                lo = mid;
            else
                hi = mid;
        }
        flag[lo] = 1;
    }
}

// Global positions of finished requests -> indices within each request.
__global__ void k_unbase(uint32_t *perm, const ReqJob *__restrict__ jobs, uint32_t njobs,
                         uint32_t total) {
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total;
         q += gridDim.x * blockDim.x) {
        const ReqJob jb = jobs[find_job(jobs, njobs, q)];
        perm[jb.pos + (q - jb.first)] -= jb.pos;
    }
}

// ---- text inputs: string starts in a delimited text ---------------------------
// The reference's sortstring turns a file into strings by create_strings_delim
// (src/sortstring.c:310-335): every delimiter byte ('\n', or NUL with --raw)
// ends one string, the next string starts right after it, text after the last
// delimiter is not a string, and '\n' delimiters are overwritten with NUL.
// Each CTA covers TEXT_TILE bytes: every thread TEXT_VEC consecutive 16-byte
// chunks, loaded together before any is examined.
constexpr int TEXT_THREADS = 256;
constexpr int TEXT_VEC = 4;
constexpr uint64_t TEXT_TILE = TEXT_THREADS * 16 * TEXT_VEC;

// Bit b of a 4-byte word's result is set when byte b equals the delimiter.
__device__ __forceinline__ uint32_t delim_bits4(uint32_t w, uint32_t d4) {
    const uint32_t t = __vcmpeq4(w, d4) & 0x01010101u;
    return (t | (t >> 7) | (t >> 14) | (t >> 21)) & 0xFu;
}

// m[c], bit b: text[base + 16 c + b] == delim (positions at or past len never
// match); the thread's chunks start at base (a multiple of 16).
__device__ __forceinline__ void delim_masks(const uint8_t *__restrict__ text, uint64_t len,
                                            uint64_t base, uint8_t delim,
                                            uint32_t (&m)[TEXT_VEC]) {
    if (base + 16 * TEXT_VEC <= len) {
        const uint32_t d4 = 0x01010101u * delim;
        uint4 v[TEXT_VEC];
#pragma unroll
        for (int c = 0; c < TEXT_VEC; ++c) v[c] = reinterpret_cast<const uint4 *>(text + base)[c];
#pragma unroll
        for (int c = 0; c < TEXT_VEC; ++c)
            m[c] = delim_bits4(v[c].x, d4) | delim_bits4(v[c].y, d4) << 4 |
                   delim_bits4(v[c].z, d4) << 8 | delim_bits4(v[c].w, d4) << 12;
    } else {
#pragma unroll
        for (int c = 0; c < TEXT_VEC; ++c) {
            m[c] = 0;
            for (uint64_t b = 0; b < 16 && base + 16 * c + b < len; ++b)
                if (text[base + 16 * c + b] == delim) m[c] |= 1u << b;
        }
    }
}

__global__ void __launch_bounds__(TEXT_THREADS)
    k_text_count(const uint8_t *__restrict__ text, uint64_t len, uint8_t delim,
                 uint32_t *tile_cnt, unsigned long long *total) {
    __shared__ uint32_t warp_sums[TEXT_THREADS / 32];
    const uint64_t base = blockIdx.x * TEXT_TILE + threadIdx.x * (16ull * TEXT_VEC);
    uint32_t m[TEXT_VEC];
    delim_masks(text, len, base, delim, m);
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < TEXT_VEC; ++q) c += __popc(m[q]);
#pragma unroll
    for (int d = 16; d; d >>= 1) c += __shfl_xor_sync(0xffffffffu, c, d);
    if ((threadIdx.x & 31) == 0) warp_sums[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < TEXT_THREADS / 32; ++w) t += warp_sums[w];
        tile_cnt[blockIdx.x] = t;
        if (t) atomicAdd(total, (unsigned long long)t);
    }
}

// tile_base: exclusive prefix of the tile counts; n: total delimiters.  String
// r + 1 starts right after delimiter r; string 0 starts at 0.
__global__ void __launch_bounds__(TEXT_THREADS)
    k_text_starts(uint8_t *text, uint64_t len, uint8_t delim, const uint32_t *__restrict__ tile_base,
                  uint64_t n, void *offs, int off_width) {
    __shared__ uint32_t warp_sums[TEXT_THREADS / 32];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint64_t base = blockIdx.x * TEXT_TILE + threadIdx.x * (16ull * TEXT_VEC);
    uint32_t m[TEXT_VEC];
    delim_masks(text, len, base, delim, m);
    uint32_t c = 0;
#pragma unroll
    for (int q = 0; q < TEXT_VEC; ++q) c += __popc(m[q]);
    uint32_t v = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= (uint32_t)d) v += y;
    }
    if (lane == 31) warp_sums[w] = v;
    __syncthreads();
    uint32_t before = 0;
    for (uint32_t q = 0; q < w; ++q) before += warp_sums[q];
    uint64_t r = (uint64_t)tile_base[blockIdx.x] + before + v - c;
#pragma unroll
    for (int q = 0; q < TEXT_VEC; ++q) {
        uint32_t mq = m[q];
        while (mq) {
            const int b = __ffs(mq) - 1;
            mq &= mq - 1;
            const uint64_t i = base + 16 * q + b;
            if (r + 1 < n) {
                if (off_width == 8)
                    static_cast<uint64_t *>(offs)[r + 1] = i + 1;
                else
                    static_cast<uint32_t *>(offs)[r + 1] = (uint32_t)(i + 1);
            }
            if (delim) text[i] = 0;
            ++r;
        }
    }
    if (blockIdx.x == 0 && threadIdx.x == 0 && n) {
        if (off_width == 8)
            static_cast<uint64_t *>(offs)[0] = 0;
        else
            static_cast<uint32_t *>(offs)[0] = 0;
    }
}

// offs[i] = i: every suffix of the text (sortstring --suffix-sorting,
// create_suffixes, src/sortstring.c:349-358).
__global__ void k_iota_offs(void *offs, int off_width, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (off_width == 8)
            static_cast<uint64_t *>(offs)[i] = i;
        else
            static_cast<uint32_t *>(offs)[i] = (uint32_t)i;
    }
}

// out[k] = offs[perm[k]]: the sorted string starts.
// out[k] = offs[perm[k]], as out_width-byte values (4 only when every
// offset fits, which the caller knows).
__global__ void k_sorted_offs(const uint32_t *__restrict__ perm, const void *offs, int off_width,
                              uint64_t n, void *out, int out_width) {
    for (uint64_t k = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; k < n;
         k += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t i = perm[k];
        const uint64_t o = off_width == 8 ? static_cast<const uint64_t *>(offs)[i]
                                          : static_cast<const uint32_t *>(offs)[i];
        if (out_width == 8)
            static_cast<uint64_t *>(out)[k] = o;
        else
            static_cast<uint32_t *>(out)[k] = (uint32_t)o;
    }
}

// ---- tuning: byte histogram of a sample of keys -----------------------------
// hist[b] += occurrences of byte value b among the first 8 key bytes of
// `samples` strings spread evenly over the n input strings (one CTA).
__global__ void k_byte_hist(const uint8_t *__restrict__ arena, uint64_t arena_bytes,
                            const void *offs, int off_width, uint32_t n, uint32_t samples,
                            uint32_t *hist) {
    __shared__ uint32_t h[256];
    for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x) h[b] = 0;
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < samples; i += blockDim.x) {
        const uint32_t id = (uint32_t)((uint64_t)i * n / samples);
        const Key k = load_key(arena, arena_bytes, string_offset(offs, off_width, id));
#pragma unroll
        for (int b = 0; b < 8; ++b) atomicAdd(&h[(k.hi >> (56 - 8 * b)) & 0xFF], 1u);
    }
    __syncthreads();
    for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = h[b];
}

// ---- single-CTA exclusive scans of short per-segment arrays -----------------
constexpr int SMALL_SCAN_THREADS = 1024;

// Inclusive scan of v across the CTA; returns the CTA total in `total`.
__device__ __forceinline__ uint32_t cta_inclusive_scan(uint32_t v, uint32_t &total,
                                                       uint32_t *warp_sums) {
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= (uint32_t)d) v += y;
    }
    if (lane == 31) warp_sums[w] = v;
    __syncthreads();
    uint32_t before = 0;
    total = 0;
    for (uint32_t q = 0; q < SMALL_SCAN_THREADS / 32; ++q) {
        const uint32_t x = warp_sums[q];
        if (q < w) before += x;
        total += x;
    }
    __syncthreads();
    return v + before;
}

// out0/out1 = exclusive scans of in0/in1 (n entries); out*[n] = totals.
__global__ void __launch_bounds__(SMALL_SCAN_THREADS) k_scan_pair(const uint32_t *__restrict__ in0,
                                                                   uint32_t *out0,
                                                                   const uint32_t *__restrict__ in1,
                                                                   uint32_t *out1, Count cnt) {
    __shared__ uint32_t warp_sums[SMALL_SCAN_THREADS / 32];
    const uint32_t n = count_of(cnt);
    uint32_t c0 = 0, c1 = 0;
    for (uint32_t b = 0; b < n; b += SMALL_SCAN_THREADS) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v0 = i < n ? in0[i] : 0, v1 = i < n ? in1[i] : 0;
        uint32_t t0, t1;
        const uint32_t s0 = cta_inclusive_scan(v0, t0, warp_sums);
        const uint32_t s1 = cta_inclusive_scan(v1, t1, warp_sums);
        if (i < n) {
            out0[i] = c0 + s0 - v0;
            out1[i] = c1 + s1 - v1;
        }
        c0 += t0;
        c1 += t1;
    }
    if (threadIdx.x == 0) {
        out0[n] = c0;
        out1[n] = c1;
    }
}

// out = exclusive scan of ceil(len / tile) over the segments; out[n] = total.
__global__ void __launch_bounds__(SMALL_SCAN_THREADS) k_seg_tiles(const Seg *__restrict__ segs,
                                                                   Count cnt, uint32_t tile,
                                                                   uint32_t *out) {
    __shared__ uint32_t warp_sums[SMALL_SCAN_THREADS / 32];
    const uint32_t n = count_of(cnt);
    uint32_t c = 0;
    for (uint32_t b = 0; b < n; b += SMALL_SCAN_THREADS) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < n ? (segs[i].len + tile - 1) / tile : 0;
        uint32_t t;
        const uint32_t s = cta_inclusive_scan(v, t, warp_sums);
        if (i < n) out[i] = c + s - v;
        c += t;
    }
    if (threadIdx.x == 0) out[n] = c;
}

// ---- exclusive scan (u32), three phases ----------------------------------
constexpr int SCAN_THREADS = 256;
constexpr int SCAN_ITEMS = 16;
constexpr int SCAN_CHUNK = SCAN_THREADS * SCAN_ITEMS;

// Block-wide exclusive scan of one value per thread; returns the block total.
__device__ __forceinline__ uint32_t block_exclusive_scan(uint32_t v, uint32_t &excl) {
    __shared__ uint32_t warp_tot[SCAN_THREADS / 32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncthreads();
    uint32_t wbase = 0, total = 0;
    for (int i = 0; i < SCAN_THREADS / 32; ++i) {
        const uint32_t t = warp_tot[i];
        if (i < w) wbase += t;
        total += t;
    }
    excl = wbase + x - v;
    __syncthreads();
    return total;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_reduce(const uint32_t *__restrict__ in,
                                                              Count cnt, uint32_t *partials) {
    const uint32_t n = count_of(cnt);
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_CHUNK;
    uint32_t s = 0;
    if (base < n) {
        for (int k = 0; k < SCAN_ITEMS; ++k) {
            const uint64_t i = base + (uint64_t)k * SCAN_THREADS + threadIdx.x;
            if (i < n) s += in[i];
        }
    }
    uint32_t excl;
    const uint32_t tot = block_exclusive_scan(s, excl);
    if (threadIdx.x == 0) partials[blockIdx.x] = tot;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_partials(uint32_t *partials,
                                                                uint32_t nparts) {
    uint32_t carry = 0;
    for (uint32_t b = 0; b < nparts; b += SCAN_THREADS) {
        const uint32_t i = b + threadIdx.x;
        const uint32_t v = i < nparts ? partials[i] : 0;
        uint32_t excl;
        const uint32_t tot = block_exclusive_scan(v, excl);
        if (i < nparts) partials[i] = carry + excl;
        carry += tot;
    }
    if (threadIdx.x == 0) partials[nparts] = carry;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_down(const uint32_t *in, uint32_t *out,
                                                            Count cnt,
                                                            const uint32_t *__restrict__ partials,
                                                            uint32_t nparts) {
    __shared__ uint32_t buf[SCAN_CHUNK];
    const uint32_t n = count_of(cnt);
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_CHUNK;
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = partials[nparts];
    if (base >= n) return;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const int j = k * SCAN_THREADS + threadIdx.x;
        const uint64_t i = base + j;
        buf[j] = i < n ? in[i] : 0;
    }
    __syncthreads();
    uint32_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) s += buf[threadIdx.x * SCAN_ITEMS + k];
    uint32_t excl;
    block_exclusive_scan(s, excl);
    uint32_t run = partials[blockIdx.x] + excl;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const int j = threadIdx.x * SCAN_ITEMS + k;
        const uint32_t v = buf[j];
        buf[j] = run;
        run += v;
    }
    __syncthreads();
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const int j = k * SCAN_THREADS + threadIdx.x;
        const uint64_t i = base + j;
        if (i < n) out[i] = buf[j];
    }
}

// ---- key gather for large segments ----------------------------------------
__global__ void __launch_bounds__(GATHER_THREADS) k_gather(SortArgs a, const Seg *__restrict__ L,
                                                          Count cnt,
                                                          const uint32_t *__restrict__ tile_base,
                                                          Counters *ctr) {
    const uint32_t nL = count_of(cnt);
    constexpr int U = GATHER_ITEMS;
    static_assert(GATHER_TILE % (GATHER_THREADS * GATHER_ITEMS) == 0, "tile shape");
    const uint32_t total_tiles = tile_base[nL] * (GATHER_TILE / (GATHER_THREADS * U));
    constexpr uint32_t SUBT = GATHER_TILE / (GATHER_THREADS * U);
    for (uint32_t t2 = blockIdx.x; t2 < total_tiles; t2 += gridDim.x) {
        const uint32_t t = t2 / SUBT;
        const uint32_t si = find_seg(tile_base, nL, t);
        const Seg s = L[si];
        const uint32_t lo = (t - tile_base[si]) * GATHER_TILE + (t2 % SUBT) * GATHER_THREADS * U;
        if (lo >= s.len) continue;
        const uint32_t *I = a.idx[0];
        // Depth 0 with a.key2: also keep key bytes 16..31 for round 1 (their
        // sectors are read here anyway); depth 16: read those copies.
        const bool save = a.key2 && s.depth == 0;
        const bool saved = a.key2 && s.depth == KEY_BYTES;
        uint32_t id[U];
        uint64_t off[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = lo + u * GATHER_THREADS + threadIdx.x;
            id[u] = i < s.len ? I[s.start + i] : IDX_MAX;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            off[u] = id[u] != IDX_MAX && !saved ? string_offset(a.offs, a.off_width, id[u]) : 0;
        uint32_t kept = 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = lo + u * GATHER_THREADS + threadIdx.x;
            if (id[u] != IDX_MAX) {
                a.key[0][s.start + i] =
                    saved ? a.key2[id[u]]
                          : from_key(load_key(a.arena, a.arena_bytes, off[u] + s.depth));
                if (save)
                    a.key2[id[u]] =
                        from_key(load_key(a.arena, a.arena_bytes, off[u] + KEY_BYTES));
                ++kept;
            }
        }
        if (save || saved) {
            const unsigned long long k = warp_sum((unsigned long long)kept);
            if ((threadIdx.x & 31) == 0 && k)
                atomicAdd(save ? &ctr->window_saved : &ctr->window_used, k);
        }
    }
}

// ---- splitter selection: one CTA per large segment ------------------------
constexpr int SAMPLE_THREADS = 512;
constexpr uint32_t SAMPLE_KEEP = 1024;  // samples kept in shared memory (16 KB)

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__device__ __forceinline__ void sample_segment(const SortArgs &a, const Seg *__restrict__ L,
                                               uint32_t si, ulonglong2 *spl, uint32_t *nspl,
                                               uint16_t *tbl, uint32_t *ntiles, uint32_t *cm_size,
                                               bool from_arena);

// One CTA per large segment at a time (segments si = blockIdx.x, + gridDim.x, ...).
__global__ void __launch_bounds__(SAMPLE_THREADS, 2) k_sample(SortArgs a, const Seg *__restrict__ L,
                                                           Count cnt, ulonglong2 *spl,
                                                           uint32_t *nspl, uint16_t *tbl,
                                                           uint32_t *ntiles, uint32_t *cm_size,
                                                           bool from_arena) {
    const uint32_t nL = count_of(cnt);
    for (uint32_t si = blockIdx.x; si < nL; si += gridDim.x) {
        sample_segment(a, L, si, spl, nspl, tbl, ntiles, cm_size, from_arena);
        __syncthreads();  // shared memory is reused by the next segment
    }
}

__device__ __forceinline__ void sample_segment(const SortArgs &a, const Seg *__restrict__ L,
                                               uint32_t si, ulonglong2 *spl, uint32_t *nspl,
                                               uint16_t *tbl, uint32_t *ntiles, uint32_t *cm_size,
                                               bool from_arena) {
    // sv: the samples' packed sort keys (padded layout).  Up to SAMPLE_KEEP
    // samples are loaded by all threads into smp and the candidates are read
    // from there; larger samples stay in registers and only the chosen
    // candidates are read again.
    extern __shared__ __align__(16) unsigned char sample_smem[];
    uint64_t *sv = reinterpret_cast<uint64_t *>(sample_smem);
    ulonglong2 *smp = reinterpret_cast<ulonglong2 *>(sv + SAMPLES_MAX + SAMPLES_MAX / 8);
    __shared__ ulonglong2 cands[SAMPLE_THREADS];
    __shared__ uint32_t warp_cnt[SAMPLE_THREADS / 32 + 1];
    __shared__ uint64_t red[4][SAMPLE_THREADS / 32];
    const Seg s = L[si];
    const ulonglong2 *K = a.keyb(s.flags & SEG_BUF1) + s.start;
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const uint32_t tcls = a.target_by_class[31 - __clz(s.len)];
    const uint32_t tb = tcls ? tcls : a.target_bucket;
    uint32_t k = (s.len + tb - 1) / tb;
    if (k > a.max_splitters) k = a.max_splitters;
    if (k < 1) k = 1;
    uint32_t S = next_pow2(8 * (k + 1));
    if (S < 256) S = 256;
    if (S > (uint32_t)SAMPLES_MAX) S = SAMPLES_MAX;
    // Sample i is the string at position pos_of(i) of the segment.  On the
    // first partition level of a round the segment's keys are not in the key
    // buffer yet (the count kernel gathers them): read them from the arena.
    auto pos_of = [&](uint32_t i) -> uint32_t {
        const uint32_t r = hash32(s.start * 0x9E3779B1u + i * 0x85EBCA77u + s.len);
        return (uint32_t)(((uint64_t)r * s.len) >> 32);
    };
    auto key_at = [&](uint32_t e) -> Key {
        return from_arena ? load_key(a.arena, a.arena_bytes,
                                     string_offset(a.offs, a.off_width, a.idx[0][s.start + e]) +
                                         s.depth)
                          : to_key(K[e]);
    };
    // Warp w < S / 256 holds samples w * 256 + lane * 8 + i (i < 8).
    const bool active = w * 256 < S;
    const bool kept = S <= SAMPLE_KEEP;  // block-uniform
    if (kept) {
        for (uint32_t i = threadIdx.x; i < S; i += SAMPLE_THREADS)
            smp[i] = from_key(key_at(pos_of(i)));
        __syncthreads();
    }
    Key kk[8];
    uint64_t oh = 0, ol = 0, ah = ~0ull, al = ~0ull;
    if (active) {
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t e = w * 256 + lane * 8 + i;
            kk[i] = kept ? to_key(smp[e]) : key_at(pos_of(e));
        }
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            oh |= kk[i].hi;
            ol |= kk[i].lo;
            ah &= kk[i].hi;
            al &= kk[i].lo;
        }
    }
    // fs: the first bit in which the samples differ (where OR and AND differ).
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        oh |= __shfl_xor_sync(0xffffffffu, oh, d);
        ol |= __shfl_xor_sync(0xffffffffu, ol, d);
        ah &= __shfl_xor_sync(0xffffffffu, ah, d);
        al &= __shfl_xor_sync(0xffffffffu, al, d);
    }
    if (lane == 0) {
        red[0][w] = oh;
        red[1][w] = ol;
        red[2][w] = ah;
        red[3][w] = al;
    }
    __syncthreads();
    uint64_t dh = 0, dl = 0;
    {
        uint64_t h1 = 0, l1 = 0, h0 = ~0ull, l0 = ~0ull;
#pragma unroll
        for (int q = 0; q < SAMPLE_THREADS / 32; ++q) {
            h1 |= red[0][q];
            l1 |= red[1][q];
            h0 &= red[2][q];
            l0 &= red[3][q];
        }
        dh = h1 ^ h0;
        dl = l1 ^ l0;
    }
    const uint32_t fs = (dh | dl) ? clz128(dh, dl) : 128u;
    // Order the samples by packed keys (window after the samples' common
    // prefix, 12-bit sample index): warp runs of 256, then merges.  The order
    // only picks quantiles; the chosen candidates are sorted by full key below.
    if (active) {
        uint64_t v[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            const uint32_t e = w * 256 + lane * 8 + i;
            v[i] = fs < 128 ? ((window64(kk[i], fs) & ~0xFFFull) | e) : e;
        }
        warp_merge_sort64<8>(v, sv, w * 256, lane);
    }
    __syncthreads();
    for (uint32_t run = 256; run < S; run <<= 1) {
        const uint32_t o = threadIdx.x * 8;
        uint64_t ov[8];
        const bool act = o < S;
        if (act) {
            const uint32_t a0 = o & ~(2 * run - 1), b0 = a0 + run;  // run: a power of two
            const uint32_t d = o - a0;
            uint32_t ia = merge_split64(sv, a0, run, b0, run, d);
            uint32_t ib = d - ia;
#pragma unroll
            for (int i = 0; i < 8; ++i) {
                const uint64_t va = ia < run ? sv[pad(a0 + ia)] : ~0ull;
                const uint64_t vb = ib < run ? sv[pad(b0 + ib)] : ~0ull;
                const bool take_a = ib >= run || (ia < run && va < vb);
                ov[i] = take_a ? va : vb;
                ia += take_a;
                ib += !take_a;
            }
        }
        __syncthreads();
        if (act) {
#pragma unroll
            for (int i = 0; i < 8; ++i) sv[pad(o + i)] = ov[i];
        }
        __syncthreads();
    }
    // Candidates at ranks (j+1)*S/(k+1), padded with the all-ones key.  They
    // are in packed-key order, which is full-key order unless two windows
    // tie; only then a bitonic network over the next power of two >= k slots
    // sorts them by full key.
    {
        const uint32_t j = threadIdx.x;
        if (j < k) {
            const uint32_t e = sv[pad(((j + 1) * S) / (k + 1))] & 0xFFF;
            cands[j] = kept ? smp[e] : from_key(key_at(pos_of(e)));
        } else {
            cands[j] = from_key(key_max());
        }
    }
    __syncthreads();
    const bool out_of_order = threadIdx.x + 1 < k &&
                              key_lt(to_key(cands[threadIdx.x + 1]), to_key(cands[threadIdx.x]));
    if (__syncthreads_or(out_of_order)) {
        const uint32_t kp = next_pow2(k);
        for (uint32_t kk = 2; kk <= kp; kk <<= 1) {
            for (uint32_t jj = kk >> 1; jj > 0; jj >>= 1) {
                const uint32_t i = threadIdx.x, l = i ^ jj;
                bool take = false;
                Key y{0, 0};
                if (i < kp) {
                    const Key x = to_key(cands[i]);
                    y = to_key(cands[l]);
                    const bool lower = l > i;
                    const bool asc = (i & kk) == 0;
                    // the lower slot keeps the min when ascending, the max otherwise
                    take = lower ? (asc ? key_lt(y, x) : key_lt(x, y))
                                 : (asc ? key_lt(x, y) : key_lt(y, x));
                }
                __syncthreads();
                if (take) cands[i] = from_key(y);
                __syncthreads();
            }
        }
    }
    // Survivors: the distinct candidates, compacted in order.
    const uint32_t j = threadIdx.x;
    Key cand{0, 0};
    bool keep = false;
    if (j < k) {
        cand = to_key(cands[j]);
        keep = j == 0 || !key_eq(to_key(cands[j - 1]), cand);
    }
    const uint32_t bal = __ballot_sync(0xffffffffu, keep);
    if (lane == 0) warp_cnt[w] = __popc(bal);
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (int q = 0; q < SAMPLE_THREADS / 32; ++q) {
            const uint32_t v = warp_cnt[q];
            warp_cnt[q] = run;
            run += v;
        }
        warp_cnt[SAMPLE_THREADS / 32] = run;
    }
    __syncthreads();
    const uint32_t u = warp_cnt[SAMPLE_THREADS / 32];
    ulonglong2 *out = spl + (uint64_t)si * SPL_STRIDE;
    if (keep) {
        const uint32_t pos = warp_cnt[w] + __popc(bal & lanemask_lt());
        out[pos] = from_key(cand);
        cands[pos] = from_key(cand);  // candidates were read before the barriers
    }
    const uint32_t kp2 = next_pow2(u + 1);
    for (uint32_t q = u + threadIdx.x; q + 1 < kp2; q += SAMPLE_THREADS)
        out[q] = from_key(key_max());
    __syncthreads();
    // Lookup table over the TBL_BITS bits after the splitters' common prefix.
    const Key s0 = to_key(cands[0]), sl = to_key(cands[u - 1]);
    const uint32_t f = u >= 2 ? clz128(s0.hi ^ sl.hi, s0.lo ^ sl.lo) : 128u;
    if (f < 128) {
        // The splitters' window bits first (non-decreasing, as the splitters
        // are sorted), into the packed-key area, which is free by now; then
        // each table entry is the number of splitters whose window bits are
        // below the entry's value (a binary search over those values).
        uint16_t *wb = reinterpret_cast<uint16_t *>(sv);
        for (uint32_t j = threadIdx.x; j < u; j += SAMPLE_THREADS)
            wb[j] = (uint16_t)window_bits(to_key(cands[j]), f);
        __syncthreads();
        // Thread t fills entries 8t .. 8t + 7 (and one more thread the last
        // entry): two searches bound the splitters of its 8 window values,
        // then each entry searches only between them.
        uint16_t *T = tbl + (uint64_t)si * TBL_STRIDE;
        auto lower = [&](uint32_t lo, uint32_t hi, uint32_t wv) -> uint32_t {
            while (lo < hi) {
                const uint32_t mid = (lo + hi) >> 1;
                if (wb[mid] < wv)
                    lo = mid + 1;
                else
                    hi = mid;
            }
            return lo;
        };
        static_assert(TBL_N == SAMPLE_THREADS * 8, "table entries per thread");
        const uint32_t w0 = threadIdx.x * 8;
        uint32_t lo = lower(0, u, w0);
        const uint32_t hi = lower(lo, u, w0 + 8);
        uint32_t tv[4];
#pragma unroll
        for (int i = 0; i < 8; i += 2) {
            const uint32_t t0 = lower(lo, hi, w0 + i);
            lo = lower(t0, hi, w0 + i + 1);
            tv[i / 2] = t0 | (lo << 16);
        }
        *reinterpret_cast<uint4 *>(T + w0) = make_uint4(tv[0], tv[1], tv[2], tv[3]);
        if (threadIdx.x == 0) T[TBL_N] = (uint16_t)lower(0, u, TBL_N);
    }
    if (threadIdx.x == 0) {
        nspl[si] = u | (f << 16);
        const uint32_t nt = (s.len + PART_TILE - 1) / PART_TILE;
        ntiles[si] = nt;
        cm_size[si] = (2 * u + 1) * nt;
    }
}

// ---- partition count: per-tile bucket histograms ---------------------------
// Each warp counts its own 512 consecutive keys into a private row, one
// shared-memory update per distinct bucket per 32 keys (__match_any_sync).
// Shared memory of the partition kernels.
struct PartSmem {
    ulonglong2 spl[SPL_STRIDE];              // the segment's splitters
    uint16_t tbl[TBL_N + 8];                 // splitter lookup table
    uint16_t cnt[PART_WARPS][NB_MAX + 1];    // per-warp bucket counters
    uint32_t gbase[NB_MAX + 1];              // tile's global base per bucket
};

// Splitters (and the lookup table when f < 128) of segment si into smem.
__device__ __forceinline__ void load_splitters(PartSmem &sm, const ulonglong2 *__restrict__ spl,
                                               const uint16_t *__restrict__ tbl, uint32_t si,
                                               uint32_t u, uint32_t f) {
    for (uint32_t q = threadIdx.x; q < u; q += PART_THREADS)
        sm.spl[q] = spl[(uint64_t)si * SPL_STRIDE + q];
    if (f < 128) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(tbl + (uint64_t)si * TBL_STRIDE);
        uint32_t *dst = reinterpret_cast<uint32_t *>(sm.tbl);
        for (uint32_t q = threadIdx.x; q < (TBL_N + 2) / 2; q += PART_THREADS) dst[q] = src[q];
    }
}

// GATHER (first partition level of a round): the keys are loaded from the
// arena through idx and offsets and stored to the key buffer here, so the
// key gather's random arena reads overlap the classification work.
template <bool GATHER>
__global__ void __launch_bounds__(PART_THREADS, 2) k_count(SortArgs a, const Seg *__restrict__ L,
                                                        Count cnt,
                                                        const uint32_t *__restrict__ tile_base,
                                                        const ulonglong2 *__restrict__ spl,
                                                        const uint32_t *__restrict__ nspl,
                                                        const uint16_t *__restrict__ tbl,
                                                        const uint32_t *__restrict__ cm_base,
                                                        uint32_t *cm, Counters *cnt_ctr) {
    extern __shared__ __align__(16) unsigned char part_smem[];
    PartSmem &sm = *reinterpret_cast<PartSmem *>(part_smem);
    auto &hist = sm.cnt;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int SUB = PART_TILE / PART_WARPS;
    const uint32_t nL = count_of(cnt);
    const uint32_t total_tiles = tile_base[nL];
    const uint32_t lt = lanemask_lt();
    uint32_t loaded = ~0u;
    for (uint32_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint32_t si = find_seg(tile_base, nL, t);
        const Seg s = L[si];
        const uint32_t u = nspl[si] & 0xFFFF, f = nspl[si] >> 16, nb = 2 * u + 1;
        const uint32_t bbits = 32 - __clz(nb);  // bucket ids are 0..nb
        if (a.l2_prefetch && threadIdx.x == 0 && t + gridDim.x < total_tiles) {
            // the keys (or, when gathering, the indices) of this CTA's next tile
            const uint32_t t2 = t + gridDim.x;
            const uint32_t s2i = find_seg(tile_base, nL, t2);
            const Seg s2 = L[s2i];
            const uint32_t lo2 = (t2 - tile_base[s2i]) * PART_TILE;
            const uint32_t len2 = min((uint32_t)PART_TILE, s2.len - lo2);
            if (GATHER)
                prefetch_l2(a.idx[0] + s2.start + lo2, (uint64_t)len2 * 4);
            else
                prefetch_l2(a.keyb(s2.flags & SEG_BUF1) + s2.start + lo2, (uint64_t)len2 * 16);
        }
        if (si != loaded) {
            load_splitters(sm, spl, tbl, si, u, f);
            loaded = si;
        }
        {
            uint32_t *h32 = reinterpret_cast<uint32_t *>(&hist[0][0]);
            for (uint32_t q = threadIdx.x; q < PART_WARPS * (NB_MAX + 1) / 2; q += PART_THREADS)
                h32[q] = 0;
        }
        __syncthreads();
        const uint32_t tl = t - tile_base[si];
        const uint32_t nt = tile_base[si + 1] - tile_base[si];
        const uint32_t lo = tl * PART_TILE + w * SUB;
        Key kk[PART_ITEMS];
        if (GATHER) {
            // round-start segments live in buffer 0
            const uint32_t *I = a.idx[0] + s.start;
            ulonglong2 *KW = a.key[0] + s.start;
            if (a.key2 && s.depth == KEY_BYTES) {
                // round 1: the keys round 0's gather kept, by string id
                uint32_t got = 0;
#pragma unroll
                for (int c = 0; c < PART_ITEMS; ++c) {
                    const uint32_t e = lo + c * 32 + lane;
                    if (e < s.len) {
                        const ulonglong2 k2 = a.key2[I[e]];
                        kk[c] = to_key(k2);
                        KW[e] = k2;
                        ++got;
                    } else {
                        kk[c] = key_max();
                    }
                }
                const unsigned long long g = warp_sum((unsigned long long)got);
                if (lane == 0 && g) atomicAdd(&cnt_ctr->window_used, g);
            } else {
                // Depth 0 with a.key2 (a fresh round gathered here): also keep
                // key bytes 16..31 for round 1, as k_gather does.
                const bool save = a.key2 && s.depth == 0;
                uint64_t off[PART_ITEMS];
#pragma unroll
                for (int c = 0; c < PART_ITEMS; ++c) {
                    const uint32_t e = lo + c * 32 + lane;
                    off[c] = e < s.len ? string_offset(a.offs, a.off_width, I[e]) + s.depth : 0;
                }
                uint32_t got = 0;
#pragma unroll
                for (int c = 0; c < PART_ITEMS; ++c) {
                    const uint32_t e = lo + c * 32 + lane;
                    if (e < s.len) {
                        kk[c] = load_key(a.arena, a.arena_bytes, off[c]);
                        KW[e] = from_key(kk[c]);
                        if (save) {
                            a.key2[I[e]] =
                                from_key(load_key(a.arena, a.arena_bytes, off[c] + KEY_BYTES));
                            ++got;
                        }
                    } else {
                        kk[c] = key_max();
                    }
                }
                if (save) {
                    const unsigned long long g = warp_sum((unsigned long long)got);
                    if (lane == 0 && g) atomicAdd(&cnt_ctr->window_saved, g);
                }
            }
        } else {
            const ulonglong2 *K = a.keyb(s.flags & SEG_BUF1) + s.start;
#pragma unroll
            for (int c = 0; c < PART_ITEMS; ++c) {
                const uint32_t e = lo + c * 32 + lane;
                kk[c] = e < s.len ? to_key(K[e]) : key_max();
            }
        }
        // Bucket and rank among the warp's earlier keys of the same bucket
        // (keys are visited in position order: the scatter stays stable).
        uint32_t br[PART_ITEMS];
#pragma unroll
        for (int c = 0; c < PART_ITEMS; ++c) {
            const uint32_t e = lo + c * 32 + lane;
            const uint32_t b = e < s.len ? classify_tbl(sm.spl, sm.tbl, u, f, kk[c]) : nb;
            const uint32_t peers =
                a.match_vote ? match_bits(b, bbits) : __match_any_sync(0xffffffffu, b);
            const uint32_t r = __popc(peers & lt);
            const uint32_t base = hist[w][b];
            __syncwarp();
            if (r == 0) hist[w][b] = (uint16_t)(base + __popc(peers));
            __syncwarp();
            br[c] = (b << 16) | (base + r);
        }
        __syncthreads();
        // Per bucket: the tile's count (to the count matrix) and each warp's
        // offset inside the tile's run of that bucket.
        for (uint32_t q = threadIdx.x; q < nb; q += PART_THREADS) {
            uint32_t run = 0;
#pragma unroll
            for (int ww = 0; ww < PART_WARPS; ++ww) {
                const uint32_t x = hist[ww][q];
                hist[ww][q] = (uint16_t)run;
                run += x;
            }
            cm[cm_base[si] + (uint64_t)q * nt + tl] = run;
        }
        __syncthreads();
        // Packed destination for the scatter: bucket << 12 | offset in the
        // tile's run of that bucket (< PART_TILE).
#pragma unroll
        for (int c = 0; c < PART_ITEMS; ++c) {
            const uint32_t e = lo + c * 32 + lane;
            if (e < s.len) {
                const uint32_t b = br[c] >> 16;
                a.bkt[s.start + e] = (b << 12) | (hist[w][b] + (br[c] & 0xFFFF));
            }
        }
        __syncthreads();
    }
}

// ---- partition scatter: a copy to precomputed destinations --------------------
// k_count left every key's bucket and its offset inside the tile's run of that
// bucket; the run's start comes from the scanned count matrix.  Tile order
// and within-tile order follow positions, so the scatter is stable.  Each
// tile is first laid out in shared memory in output order (its bucket runs
// back to back), so consecutive threads store to consecutive addresses within
// every run.
constexpr int SCATTER_THREADS = 256;  // 512 x 8 items measured slower
constexpr int SCATTER_ITEMS = PART_TILE / SCATTER_THREADS;  // 16
struct ScatterSmem {
    ulonglong2 key[PART_TILE];
    uint32_t idx[PART_TILE];
    uint32_t dst[PART_TILE];
    uint32_t gbase[NB_MAX + 1];
    uint32_t tstart[NB_MAX + 1];
    uint32_t wsum[SCATTER_THREADS / 32];
};

// BULK: each bucket run of keys leaves shared memory as one asynchronous bulk
// copy to global memory (cp.async.bulk, issued by the thread that owns the
// bucket; keys are 16 bytes, so every run starts and ends on a 16-byte
// boundary at both ends); the indices are stored by the threads as before.
template <bool BULK>
__global__ void __launch_bounds__(SCATTER_THREADS) k_scatter(SortArgs a, const Seg *__restrict__ L,
                                                             Count cnt,
                                                             const uint32_t *__restrict__ tile_base,
                                                             const uint32_t *__restrict__ nspl,
                                                             const uint32_t *__restrict__ cm_base,
                                                             const uint32_t *__restrict__ cm_scan) {
    extern __shared__ __align__(16) unsigned char scatter_smem[];
    ScatterSmem &sm = *reinterpret_cast<ScatterSmem *>(scatter_smem);
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr uint32_t QPT = (NB_MAX + 1) / SCATTER_THREADS;  // buckets per thread (4)
    const uint32_t nL = count_of(cnt);
    const uint32_t total_tiles = tile_base[nL];
    bool any_bulk = false;  // this thread issued bulk copies (BULK)
    for (uint32_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint32_t si = find_seg(tile_base, nL, t);
        const Seg s = L[si];
        const uint32_t u = nspl[si] & 0xFFFF, nb = 2 * u + 1;
        if (a.l2_prefetch && threadIdx.x == 0 && t + gridDim.x < total_tiles) {
            // keys, indices and destinations of this CTA's next tile
            const uint32_t t2 = t + gridDim.x;
            const uint32_t s2i = find_seg(tile_base, nL, t2);
            const Seg s2 = L[s2i];
            const uint32_t lo2 = (t2 - tile_base[s2i]) * PART_TILE;
            const uint32_t len2 = min((uint32_t)PART_TILE, s2.len - lo2);
            const int b2 = s2.flags & SEG_BUF1;
            prefetch_l2(a.keyb(b2) + s2.start + lo2, (uint64_t)len2 * 16);
            prefetch_l2(a.idxb(b2) + s2.start + lo2, (uint64_t)len2 * 4);
            prefetch_l2(a.bkt + s2.start + lo2, (uint64_t)len2 * 4);
        }
        const uint32_t tl = t - tile_base[si];
        const uint32_t nt = tile_base[si + 1] - tile_base[si];
        const uint32_t cmb = cm_base[si];
        const uint32_t seg0 = cm_scan[cmb];
        const uint32_t lo = tl * PART_TILE;
        const uint32_t tlen = min((uint32_t)PART_TILE, s.len - lo);
        const int ib = s.flags & SEG_BUF1;
        const ulonglong2 *Kin = a.keyb(ib) + s.start;
        const uint32_t *Iin = a.idxb(ib) + s.start;
        const uint32_t *Din = a.bkt + s.start;
        // Element loads first (they overlap the count-matrix reads below).
        ulonglong2 kk[SCATTER_ITEMS];
        uint32_t ii[SCATTER_ITEMS], dd[SCATTER_ITEMS];
#pragma unroll
        for (int c = 0; c < SCATTER_ITEMS; ++c) {
            const uint32_t e = c * SCATTER_THREADS + threadIdx.x;
            if (e < tlen) {
                kk[c] = Kin[lo + e];
                ii[c] = Iin[lo + e];
                dd[c] = Din[lo + e];
            }
        }
        // Per bucket: the tile's run start in the segment and the tile's
        // count (difference of consecutive scanned entries), then an exclusive
        // scan of the counts gives each run's start inside the tile.
        uint32_t cnt[QPT];
        uint32_t mysum = 0;
#pragma unroll
        for (uint32_t j = 0; j < QPT; ++j) {
            const uint32_t q = threadIdx.x * QPT + j;
            uint32_t c0 = 0;
            if (q < nb) {
                const uint64_t at = cmb + (uint64_t)q * nt + tl;
                const uint32_t g = cm_scan[at];
                c0 = cm_scan[at + 1] - g;  // next tile, or next bucket's first tile
                sm.gbase[q] = g - seg0;
            }
            cnt[j] = c0;
            mysum += c0;
        }
        uint32_t incl = mysum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        if (lane == 31) sm.wsum[w] = incl;
        __syncthreads();
        uint32_t run = incl - mysum;
        for (uint32_t q = 0; q < w; ++q) run += sm.wsum[q];
#pragma unroll
        for (uint32_t j = 0; j < QPT; ++j) {
            sm.tstart[threadIdx.x * QPT + j] = run;
            run += cnt[j];
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < SCATTER_ITEMS; ++c) {
            const uint32_t e = c * SCATTER_THREADS + threadIdx.x;
            if (e < tlen) {
                const uint32_t b = dd[c] >> 12, off = dd[c] & (PART_TILE - 1);
                const uint32_t slot = sm.tstart[b] + off;
                sm.key[slot] = kk[c];
                sm.idx[slot] = ii[c];
                sm.dst[slot] = sm.gbase[b] + off;
            }
        }
        __syncthreads();
        ulonglong2 *Kout = a.keyb(ib ^ 1) + s.start;
        uint32_t *Iout = a.idxb(ib ^ 1) + s.start;
        if constexpr (BULK) {
            // The staged keys were written by other threads through the
            // generic proxy; make them visible to the bulk copies' async proxy.
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
            bool issued = false;
#pragma unroll
            for (uint32_t j = 0; j < QPT; ++j) {
                const uint32_t q = threadIdx.x * QPT + j;
                if (cnt[j]) {
                    const uint32_t src =
                        (uint32_t)__cvta_generic_to_shared(&sm.key[sm.tstart[q]]);
                    asm volatile(
                        "cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;" ::"l"(
                            Kout + sm.gbase[q]),
                        "r"(src), "r"(cnt[j] * 16u)
                        : "memory");
                    issued = true;
                }
            }
            if (issued) asm volatile("cp.async.bulk.commit_group;" ::: "memory");
            for (uint32_t i = threadIdx.x; i < tlen; i += SCATTER_THREADS)
                Iout[sm.dst[i]] = sm.idx[i];
            // The next tile restages into sm.key: wait until the copies have
            // read it (their global writes complete by the kernel's end).
            if (issued) asm volatile("cp.async.bulk.wait_group.read 0;" ::: "memory");
            any_bulk |= issued;
        } else {
            for (uint32_t i = threadIdx.x; i < tlen; i += SCATTER_THREADS) {
                const uint32_t o = sm.dst[i];
                Kout[o] = sm.key[i];
                Iout[o] = sm.idx[i];
            }
        }
        __syncthreads();
    }
    // Every bulk copy's writes complete before the thread exits.
    if (BULK && any_bulk) asm volatile("cp.async.bulk.wait_group 0;" ::: "memory");
}


// The same scatter with only indices and destinations staged: the slots of
// the tile in output order record where each record sits in the tile, and
// the write-out reads the keys from there (the tile was just read, and with
// SortArgs::l2_prefetch also streamed into L2 ahead; the reads stay inside
// the tile's 64 KB).  48 KB of shared memory and about half the registers of
// k_scatter, so three or four CTAs share an SM instead of two.
struct Scatter2Smem {
    uint32_t idx[PART_TILE];    // indices in output order
    uint32_t dst[PART_TILE];    // destinations in output order
    uint16_t src[PART_TILE];    // tile position of the record at each output slot
    uint32_t gbase[NB_MAX + 1];
    uint32_t tstart[NB_MAX + 1];
    uint32_t wsum[SCATTER_THREADS / 32];
};
constexpr int SCATTER2_BATCH = 4;  // keys in flight per thread in the write-out

__global__ void __launch_bounds__(SCATTER_THREADS, 3) k_scatter2(
    SortArgs a, const Seg *__restrict__ L, Count cnt, const uint32_t *__restrict__ tile_base,
    const uint32_t *__restrict__ nspl, const uint32_t *__restrict__ cm_base,
    const uint32_t *__restrict__ cm_scan) {
    extern __shared__ __align__(16) unsigned char scatter_smem[];
    Scatter2Smem &sm = *reinterpret_cast<Scatter2Smem *>(scatter_smem);
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr uint32_t QPT = (NB_MAX + 1) / SCATTER_THREADS;  // buckets per thread (4)
    const uint32_t nL = count_of(cnt);
    const uint32_t total_tiles = tile_base[nL];
    for (uint32_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint32_t si = find_seg(tile_base, nL, t);
        const Seg s = L[si];
        const uint32_t u = nspl[si] & 0xFFFF, nb = 2 * u + 1;
        if (a.l2_prefetch && threadIdx.x == 0 && t + gridDim.x < total_tiles) {
            const uint32_t t2 = t + gridDim.x;
            const uint32_t s2i = find_seg(tile_base, nL, t2);
            const Seg s2 = L[s2i];
            const uint32_t lo2 = (t2 - tile_base[s2i]) * PART_TILE;
            const uint32_t len2 = min((uint32_t)PART_TILE, s2.len - lo2);
            const int b2 = s2.flags & SEG_BUF1;
            prefetch_l2(a.keyb(b2) + s2.start + lo2, (uint64_t)len2 * 16);
            prefetch_l2(a.idxb(b2) + s2.start + lo2, (uint64_t)len2 * 4);
            prefetch_l2(a.bkt + s2.start + lo2, (uint64_t)len2 * 4);
        }
        const uint32_t tl = t - tile_base[si];
        const uint32_t nt = tile_base[si + 1] - tile_base[si];
        const uint32_t cmb = cm_base[si];
        const uint32_t seg0 = cm_scan[cmb];
        const uint32_t lo = tl * PART_TILE;
        const uint32_t tlen = min((uint32_t)PART_TILE, s.len - lo);
        const int ib = s.flags & SEG_BUF1;
        const ulonglong2 *__restrict__ Kin = a.keyb(ib) + s.start + lo;
        const uint32_t *Iin = a.idxb(ib) + s.start;
        const uint32_t *Din = a.bkt + s.start;
        uint32_t ii[SCATTER_ITEMS], dd[SCATTER_ITEMS];
#pragma unroll
        for (int c = 0; c < SCATTER_ITEMS; ++c) {
            const uint32_t e = c * SCATTER_THREADS + threadIdx.x;
            if (e < tlen) {
                ii[c] = Iin[lo + e];
                dd[c] = Din[lo + e];
            }
        }
        uint32_t cnt4[QPT];
        uint32_t mysum = 0;
#pragma unroll
        for (uint32_t j = 0; j < QPT; ++j) {
            const uint32_t q = threadIdx.x * QPT + j;
            uint32_t c0 = 0;
            if (q < nb) {
                const uint64_t at = cmb + (uint64_t)q * nt + tl;
                const uint32_t g = cm_scan[at];
                c0 = cm_scan[at + 1] - g;
                sm.gbase[q] = g - seg0;
            }
            cnt4[j] = c0;
            mysum += c0;
        }
        uint32_t incl = mysum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (uint32_t)d) incl += y;
        }
        if (lane == 31) sm.wsum[w] = incl;
        __syncthreads();
        uint32_t run = incl - mysum;
        for (uint32_t q = 0; q < w; ++q) run += sm.wsum[q];
#pragma unroll
        for (uint32_t j = 0; j < QPT; ++j) {
            sm.tstart[threadIdx.x * QPT + j] = run;
            run += cnt4[j];
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < SCATTER_ITEMS; ++c) {
            const uint32_t e = c * SCATTER_THREADS + threadIdx.x;
            if (e < tlen) {
                const uint32_t b = dd[c] >> 12, off = dd[c] & (PART_TILE - 1);
                const uint32_t slot = sm.tstart[b] + off;
                sm.src[slot] = (uint16_t)e;
                sm.idx[slot] = ii[c];
                sm.dst[slot] = sm.gbase[b] + off;
            }
        }
        __syncthreads();
        ulonglong2 *Kout = a.keyb(ib ^ 1) + s.start;
        uint32_t *Iout = a.idxb(ib ^ 1) + s.start;
        for (uint32_t i0 = 0; i0 < tlen; i0 += SCATTER2_BATCH * SCATTER_THREADS) {
            ulonglong2 kv[SCATTER2_BATCH];
#pragma unroll
            for (int q = 0; q < SCATTER2_BATCH; ++q) {
                const uint32_t i = i0 + q * SCATTER_THREADS + threadIdx.x;
                if (i < tlen) kv[q] = __ldg(Kin + sm.src[i]);
            }
#pragma unroll
            for (int q = 0; q < SCATTER2_BATCH; ++q) {
                const uint32_t i = i0 + q * SCATTER_THREADS + threadIdx.x;
                if (i < tlen) {
                    const uint32_t o = sm.dst[i];
                    Kout[o] = kv[q];
                    Iout[o] = sm.idx[i];
                }
            }
        }
        __syncthreads();
    }
}

// ---- bucket emission: one CTA per partitioned segment ----------------------
__global__ void k_emit(SortArgs a, const Seg *__restrict__ L, Count cnt,
                       const uint32_t *__restrict__ tile_base,
                       const uint32_t *__restrict__ nspl, const uint32_t *__restrict__ cm_base,
                       const uint32_t *__restrict__ cm_scan, Seg *W1, Seg *W8, SmallLists S,
                       Seg *L2, Seg *E, uint2 *B, Seg *N, Counters *c) {
    const uint32_t nL = count_of(cnt);
    for (uint32_t si = blockIdx.x; si < nL; si += gridDim.x) {
    const Seg s = L[si];
    const uint32_t u = nspl[si] & 0xFFFF, nb = 2 * u + 1;
    const uint32_t nt = tile_base[si + 1] - tile_base[si];
    const uint32_t cmb = cm_base[si];
    const uint32_t seg0 = cm_scan[cmb];
    const uint32_t ob = (s.flags & SEG_BUF1) ^ 1u;
    const uint32_t flags = ob | SEG_KEYS;
    // Uniform trip count: every warp reaches the collective appends.
    for (uint32_t b0 = 0; b0 < nb; b0 += blockDim.x) {
        const uint32_t b = b0 + threadIdx.x;
        uint32_t off = 0, len = 0;
        if (b < nb) {
            off = cm_scan[cmb + (uint64_t)b * nt] - seg0;
            const uint32_t end =
                b + 1 < nb ? cm_scan[cmb + (uint64_t)(b + 1) * nt] - seg0 : s.len;
            len = end - off;
        }
        const uint32_t p = s.start + off;
        const bool bnd = len > 0 && off > 0;
        if (len == 1 && ob) {
            a.idx[0][p] = a.idx[1][p];
            a.key[0][p] = a.key[1][p];
        }
        const bool multi = len > 1;
        const bool eq = multi && (b & 1);
        bool direct = false;
        uint32_t nch = 0;
        if (eq) {
            const Key k = to_key(a.keyb(ob)[p]);
            // In buffer 0 with its keys and not final: straight to the next round.
            direct = !ob && !key_is_end(k);
            if (!direct) nch = (len + EQ_TILE - 1) / EQ_TILE;
        }
        // Every list reservation of the bucket is issued before any result
        // is used (boundary, next round, equality work items here; the
        // length-selected lists in append_by_length).
        const WarpRes rb = warp_reserve(&c->n_bound, bnd), rn = warp_reserve(&c->n_next, direct);
        // nch equality work items per bucket: warp-level exclusive sum.
        uint32_t incl = nch;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, incl, d);
            if ((threadIdx.x & 31) >= (uint32_t)d) incl += y;
        }
        const uint32_t tot = __shfl_sync(0xffffffffu, incl, 31);
        uint32_t ebase = 0;
        if ((threadIdx.x & 31) == 31 && tot) ebase = atomicAdd(&c->n_equal, tot);
        const bool rng = multi && !(b & 1);
        append_by_length(Seg{p, len, s.depth, flags}, rng, a.warp8_cap, W1, W8, S, L2,
                         &c->n_large_next, c);
        const uint32_t tb = warp_slot(rb), tn = warp_slot(rn);
        if (bnd) B[tb] = make_uint2(p, s.depth);
        if (direct) N[tn] = Seg{p, len, s.depth + KEY_BYTES, 0u};
        ebase = __shfl_sync(0xffffffffu, ebase, 31) + incl - nch;
        for (uint32_t ch = 0; ch < nch; ++ch)
            E[ebase + ch] = Seg{p, len, s.depth, ob | (ch << SEG_CHUNK_SHIFT)};
    }
    if (threadIdx.x == 0) atomicAdd(&c->partitioned, (unsigned long long)s.len);
    }
}

// ---- segments of <= 32 strings: one warp, one string per lane -------------
constexpr int WARP_THREADS = 256;

__device__ __forceinline__ void load_elem(const SortArgs &a, const Seg &s, uint32_t e, Key &k,
                                          uint32_t &id) {
    const int b = s.flags & SEG_BUF1;
    id = a.idxb(b)[s.start + e];
    k = (s.flags & SEG_KEYS)
            ? to_key(a.keyb(b)[s.start + e])
            : load_key(a.arena, a.arena_bytes, string_offset(a.offs, a.off_width, id) + s.depth);
}

// Order of records in the in-warp refinement: run head first, then (key,
// index).  Records outside runs carry their own lane as head.
__device__ __forceinline__ bool run_lt(uint32_t h1, const Key &k1, uint32_t i1, uint32_t h2,
                                       const Key &k2, uint32_t i2) {
    return h1 != h2 ? h1 < h2 : pair_lt(k1, i1, k2, i2);
}

// Runs of exactly two strings, resolved by the whole warp: lane j compares the
// two strings' 16-byte windows at depth + 16 j, so one step covers 512 bytes;
// the first lane whose windows differ or end decides order and LCP (what a
// lane past the end of a string reads is never used).  A pair still equal
// after PAIR_CHUNKS steps stays a run, 512 * PAIR_CHUNKS bytes deeper.
// `start` is the lane's group's segment start; a pair's members keep
// ascending indices (their order when equal).  Warp-collective.
constexpr uint32_t PAIR_CHUNKS = 16;

template <int W>
__device__ __forceinline__ void warp1_pairs(const uint8_t *__restrict__ arena,
                                            uint64_t arena_bytes, const void *__restrict__ offs,
                                            int off_width, uint32_t *__restrict__ idx0,
                                            uint32_t *__restrict__ lcp, uint32_t start,
                                            uint32_t lane, uint32_t id, bool &run, uint32_t &h,
                                            uint32_t &depth, uint32_t &moved) {
    const uint32_t li = lane & (W - 1);
    const uint32_t nh1 = __shfl_down_sync(0xffffffffu, h, 1);
    const uint32_t nh2 = __shfl_down_sync(0xffffffffu, h, 2);
    const bool nr1 = __shfl_down_sync(0xffffffffu, (int)run, 1) != 0;
    const bool nr2 = __shfl_down_sync(0xffffffffu, (int)run, 2) != 0;
    const bool pair_head = run && h == lane && li + 1 < (uint32_t)W && nr1 && nh1 == h &&
                           !(li + 2 < (uint32_t)W && nr2 && nh2 == h);
    uint32_t pairs = __ballot_sync(0xffffffffu, pair_head);
    while (pairs) {
        const uint32_t p = __ffs(pairs) - 1;
        pairs &= pairs - 1;
        const uint32_t ia = __shfl_sync(0xffffffffu, id, p);
        const uint32_t ib = __shfl_sync(0xffffffffu, id, p + 1);
        const uint32_t d0 = __shfl_sync(0xffffffffu, depth, p);
        const uint32_t pos = __shfl_sync(0xffffffffu, start, p) + (p & (W - 1));
        const uint64_t oa = string_offset(offs, off_width, ia);
        const uint64_t ob = string_offset(offs, off_width, ib);
        uint32_t chunk = 0, found = 0;
        for (; chunk < PAIR_CHUNKS; ++chunk) {
            const uint64_t at = (uint64_t)d0 + chunk * (32u * KEY_BYTES) + lane * KEY_BYTES;
            const Key ka = load_key(arena, arena_bytes, oa + at);
            const Key kb = load_key(arena, arena_bytes, ob + at);
            const bool same = key_eq(ka, kb);
            const uint32_t stop = __ballot_sync(0xffffffffu, !same || key_is_end(ka));
            if (stop) {
                const uint32_t f = __ffs(stop) - 1;
                if (lane == f) {
                    const uint32_t base_d = (uint32_t)at;
                    const bool swap = !same && key_lt(kb, ka);
                    idx0[pos] = swap ? ib : ia;
                    idx0[pos + 1] = swap ? ia : ib;
                    lcp[pos + 1] = base_d + (same ? key_len(ka) : key_lcp(ka, kb));
                }
                found = 1;
                break;
            }
        }
        if (lane == p || lane == p + 1) {
            if (found) {
                run = false;
                h = lane;
            } else {
                depth += PAIR_CHUNKS * 32u * KEY_BYTES;
            }
        }
        if (lane == p) moved += 2 * (chunk + found);
    }
}

// In-warp refinement of the runs a one-per-lane sort left (lanes with `run`,
// h = the run's first lane, keys equal up to `depth`, id = the lane's record).
// Each step first resolves the runs of two with the whole warp (warp1_pairs);
// then the members of the other runs load their next 16 bytes, each run is
// re-sorted inside its own lanes, the LCPs decided at this depth are written,
// and the runs of equal keys that remain become the next step's runs.  At
// most `steps` steps, then what is left goes to the next round.  This is the
// next round's one-warp sort of those runs done without a round trip: the
// same order and LCPs.  The keys of the segment's first and last position,
// which the round's boundary pass reads, stay as the first sort wrote them.
// Returns this lane's count of string steps (for the statistics).
// Warp-collective.
template <int W>
__device__ __forceinline__ uint32_t warp1_deepen(const uint8_t *__restrict__ arena,
                                              uint64_t arena_bytes, const void *__restrict__ offs,
                                              int off_width, uint32_t *__restrict__ idx0,
                                              uint32_t *__restrict__ lcp, uint32_t steps,
                                              uint32_t start, uint32_t depth, uint32_t lane,
                                              uint32_t id, bool run, uint32_t h, Seg *N,
                                              Counters *c) {
    const uint32_t li = lane & (W - 1), base = lane & ~(uint32_t)(W - 1);
    const uint32_t m = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
    uint32_t moved = 0;
    Key k = key_max();  // records outside runs are never compared by key
    for (uint32_t it = 0; it < steps && __any_sync(0xffffffffu, run); ++it) {
        warp1_pairs<W>(arena, arena_bytes, offs, off_width, idx0, lcp, start, lane, id, run, h,
                       depth, moved);
        if (!__any_sync(0xffffffffu, run)) break;
        if (run) k = load_key(arena, arena_bytes, string_offset(offs, off_width, id) + depth);
        moved += run;
        // Sorting by (head, key, index) keeps every record outside a run in
        // its lane and every run inside its own lanes.
        uint32_t hh = run ? h : lane;
        bool r = run;
#pragma unroll
        for (int kk = 2; kk <= W; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                Key ok;
                ok.hi = __shfl_xor_sync(0xffffffffu, k.hi, j);
                ok.lo = __shfl_xor_sync(0xffffffffu, k.lo, j);
                const uint32_t oi = __shfl_xor_sync(0xffffffffu, id, j);
                const uint32_t oh = __shfl_xor_sync(0xffffffffu, hh, j);
                const bool orr = __shfl_xor_sync(0xffffffffu, (int)r, j) != 0;
                const bool up = kk == W || (lane & kk) == 0;
                const bool keep_min = ((lane & j) == 0) == up;
                const bool take = keep_min ? run_lt(oh, ok, oi, hh, k, id)
                                           : run_lt(hh, k, id, oh, ok, oi);
                if (take) {
                    k = ok;
                    id = oi;
                    hh = oh;
                    r = orr;
                }
            }
        }
        Key prev, next;
        prev.hi = __shfl_up_sync(0xffffffffu, k.hi, 1);
        prev.lo = __shfl_up_sync(0xffffffffu, k.lo, 1);
        next.hi = __shfl_down_sync(0xffffffffu, k.hi, 1);
        next.lo = __shfl_down_sync(0xffffffffu, k.lo, 1);
        const uint32_t ph = __shfl_up_sync(0xffffffffu, hh, 1);
        const uint32_t nh = __shfl_down_sync(0xffffffffu, hh, 1);
        // A run's head is one of its members' lanes, never another record's
        // own lane, so equal heads mean the same run.
        const bool same_prev = r && li > 0 && ph == hh;
        const bool same_next = r && li + 1 < (uint32_t)W && nh == hh;
        const bool eqp = same_prev && key_eq(prev, k);
        const bool eqn = same_next && key_eq(next, k);
        if (r) {
            const uint32_t p = start + li;
            idx0[p] = id;
            if (same_prev) {
                if (!eqp)
                    lcp[p] = depth + key_lcp(prev, k);
                else if (key_is_end(k))
                    lcp[p] = depth + key_len(k);
            }
        }
        run = r && !key_is_end(k) && (eqp || eqn);
        const uint32_t heads = __ballot_sync(0xffffffffu, run && !eqp);
        h = run ? 31 - __clz(heads & m) : lane;
        depth += KEY_BYTES;
    }
    // What is still unresolved goes to the next round at the depth reached.
    const uint32_t nh = __shfl_down_sync(0xffffffffu, h, 1);
    const bool nrun = __shfl_down_sync(0xffffffffu, (int)run, 1) != 0;
    const bool tail = run && !(li + 1 < (uint32_t)W && nrun && nh == h);
    emit_next_warp(N, c, tail, start + (h - base), lane - h + 1, depth);
    return moved;
}

// Sorts one segment of at most W strings held by the W lanes of one aligned
// lane group (W = 8 or 32; lane li of the group holds string li).  Every
// lane of the warp calls this with its group's segment (len 0 for idle
// groups): the shuffles, ballots and the next-round append are
// warp-collective.
template <int W>
__device__ __forceinline__ uint32_t warp1_group(const SortArgs &a, const Seg &s, uint32_t lane,
                                                Seg *N, Counters *c) {
    const uint32_t li = lane & (W - 1), base = lane & ~(uint32_t)(W - 1);
    const bool v = li < s.len;
    uint32_t id = IDX_MAX;
    Key k = key_max();
    if (v) load_elem(a, s, li, k, id);
    // Bits in which the group's keys differ.
    Key k0;
    k0.hi = __shfl_sync(0xffffffffu, k.hi, base);
    k0.lo = __shfl_sync(0xffffffffu, k.lo, base);
    uint64_t dh = v ? (k.hi ^ k0.hi) : 0, dl = v ? (k.lo ^ k0.lo) : 0;
#pragma unroll
    for (int d = W / 2; d > 0; d >>= 1) {
        dh |= __shfl_xor_sync(0xffffffffu, dh, d);
        dl |= __shfl_xor_sync(0xffffffffu, dl, d);
    }
    // Packed 64-bit keys (window after the common prefix, source lane), a
    // bitonic sort inside the group (the last stage ascending for every
    // group), then each record moves to its rank.  Groups whose keys are all
    // equal sort by lane alone, which keeps them in place.
    const bool diff = (dh | dl) != 0;
    const uint32_t f = diff ? clz128(dh, dl) : 0u;
    bool bad = false;
    if (__any_sync(0xffffffffu, diff)) {  // else every group's keys are all equal
        uint64_t x = !v ? ~0ull : (diff ? sort_key(k, f, lane) : (uint64_t)lane);
#pragma unroll
        for (int kk = 2; kk <= W; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                const uint64_t y = __shfl_xor_sync(0xffffffffu, x, j);
                const bool up = kk == W || (lane & kk) == 0;
                const bool keep_min = ((lane & j) == 0) == up;
                x = keep_min ? (y < x ? y : x) : (y < x ? x : y);
            }
        }
        const uint32_t src = v ? (uint32_t)(x & 31) : lane;
        Key kn;
        kn.hi = __shfl_sync(0xffffffffu, k.hi, src);
        kn.lo = __shfl_sync(0xffffffffu, k.lo, src);
        const uint32_t idn = __shfl_sync(0xffffffffu, id, src);
        k = kn;
        id = idn;
        // Pairs with equal windows must also be in full-key order.
        Key kp;
        kp.hi = __shfl_up_sync(0xffffffffu, k.hi, 1);
        kp.lo = __shfl_up_sync(0xffffffffu, k.lo, 1);
        bad = v && diff && li > 0 &&
              (window64(kp, f) >> POS_BITS) == (window64(k, f) >> POS_BITS) && key_lt(k, kp);
    }
    if (__any_sync(0xffffffffu, bad)) {
        // Full (key, index) comparator over every group (rare).
#pragma unroll
        for (int kk = 2; kk <= W; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                Key ok;
                ok.hi = __shfl_xor_sync(0xffffffffu, k.hi, j);
                ok.lo = __shfl_xor_sync(0xffffffffu, k.lo, j);
                const uint32_t oi = __shfl_xor_sync(0xffffffffu, id, j);
                const bool up = kk == W || (lane & kk) == 0;
                const bool keep_min = ((lane & j) == 0) == up;
                const bool take = keep_min ? pair_lt(ok, oi, k, id) : pair_lt(k, id, ok, oi);
                if (take) {
                    k = ok;
                    id = oi;
                }
            }
        }
    }
    Key prev, next;
    prev.hi = __shfl_up_sync(0xffffffffu, k.hi, 1);
    prev.lo = __shfl_up_sync(0xffffffffu, k.lo, 1);
    next.hi = __shfl_down_sync(0xffffffffu, k.hi, 1);
    next.lo = __shfl_down_sync(0xffffffffu, k.lo, 1);
    const bool head = v && (li == 0 || !key_eq(prev, k));
    const uint32_t heads = __ballot_sync(0xffffffffu, head);
    if (v) {
        const uint32_t p = s.start + li;
        a.idx[0][p] = id;
        if (li == 0 || li == s.len - 1) a.key[0][p] = from_key(k);
        if (li > 0) {
            if (!key_eq(prev, k))
                a.lcp[p] = s.depth + key_lcp(prev, k);
            else if (key_is_end(k))
                a.lcp[p] = s.depth + key_len(k);
        }
    }
    // Runs: maximal groups of at least two equal keys that do not end; h is
    // the run's first lane (at or after the group's lane 0).
    const bool eq_next = v && li + 1 < s.len && key_eq(next, k);
    bool run = v && !key_is_end(k) && (!head || eq_next);
    const uint32_t m = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
    uint32_t h = run ? 31 - __clz(heads & m) : lane;
    if (a.warp1_deep && __any_sync(0xffffffffu, run))
        return warp1_deepen<W>(a.arena, a.arena_bytes, a.offs, a.off_width, a.idx[0], a.lcp,
                               a.warp1_deep, s.start, s.depth + KEY_BYTES, lane, id, run, h, N,
                               c);
    const bool tail = run && !eq_next;  // a run's last lane
    emit_next_warp(N, c, tail, s.start + (h - base), lane - h + 1, s.depth + KEY_BYTES);
    return 0;
}

// Segments of <= WARP1_CAP strings.  First pass: a warp takes W1_PACK
// consecutive list entries and sorts those of at most 8 strings together, one
// per 8-lane group, so that their loads overlap.  Second pass: one warp per
// remaining segment.
constexpr uint32_t W1_PACK = 4;

__global__ void __launch_bounds__(WARP_THREADS) k_warp1(SortArgs a, const Seg *__restrict__ T0,
                                                        Span sp, Seg *N, Counters *c) {
    const uint32_t lo = count_of(sp.lo);
    const Seg *__restrict__ T = T0 + lo;
    const uint32_t nT = count_of(sp.hi) - lo;
    const uint32_t lane = threadIdx.x & 31;
    const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long fresh = 0, keyed = 0, deep = 0;
    for (uint32_t g0 = warp0 * W1_PACK; g0 < nT; g0 += nwarps * W1_PACK) {
        const uint32_t j = lane >> 3;
        const Seg sj = g0 + j < nT ? T[g0 + j] : Seg{0, 0, 0, 0};
        const bool small = sj.len <= 8;
        if ((lane & 7) == 0) {
            if (sj.flags & SEG_KEYS)
                keyed += sj.len;
            else
                fresh += sj.len;
        }
        if (__any_sync(0xffffffffu, small && sj.len > 0))
            deep += warp1_group<8>(a, small ? sj : Seg{0, 0, 0, 0}, lane, N, c);
    }
    for (uint32_t g = warp0; g < nT; g += nwarps) {
        const Seg s = T[g];
        if (s.len > 8) deep += warp1_group<32>(a, s, lane, N, c);
    }
    if ((lane & 7) == 0 && (fresh | keyed)) {  // each 8-lane group's leader
        atomicAdd(&c->warp1_fresh, fresh);
        atomicAdd(&c->warp1_keyed, keyed);
    }
    deep = warp_sum(deep);
    if (lane == 0 && deep) atomicAdd(&c->warp1_deep, deep);
}

// Warp-wide OR of key ^ key0 over the records at padded positions 0..len-1.
__device__ __forceinline__ uint32_t warp_diff_bit(const ulonglong2 *sk, uint32_t len,
                                                  uint32_t lane) {
    const Key k0 = to_key(sk[pad(0)]);
    uint64_t dh = 0, dl = 0;
    for (uint32_t e = lane; e < len; e += 32) {
        const Key k = to_key(sk[pad(e)]);
        dh |= k.hi ^ k0.hi;
        dl |= k.lo ^ k0.lo;
    }
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) {
        dh |= __shfl_xor_sync(0xffffffffu, dh, d);
        dl |= __shfl_xor_sync(0xffffffffu, dl, d);
    }
    return (dh | dl) ? clz128(dh, dl) : 128u;
}

// ---- segments of 33..256 strings: one warp, 2/4/8 strings per lane ----------
constexpr int W8_PAD = WARP8_CAP + WARP8_CAP / 8;
constexpr int W8_WARPS = WARP_THREADS / 32;
constexpr size_t W8_SMEM = (size_t)W8_WARPS * W8_PAD * (sizeof(ulonglong2) + sizeof(uint64_t) +
                                                         sizeof(uint32_t));

__global__ void __launch_bounds__(WARP_THREADS, 3) k_warp8(SortArgs a, const Seg *__restrict__ T0,
                                                           Span sp, Seg *N, Counters *c) {
    const uint32_t lo = count_of(sp.lo);
    const Seg *__restrict__ T = T0 + lo;
    const uint32_t nT = count_of(sp.hi) - lo;
    extern __shared__ __align__(16) unsigned char w8_smem[];
    const uint32_t lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    ulonglong2 *sk = reinterpret_cast<ulonglong2 *>(w8_smem) + w * W8_PAD;
    uint64_t *sv = reinterpret_cast<uint64_t *>(reinterpret_cast<ulonglong2 *>(w8_smem) +
                                                W8_WARPS * W8_PAD) + w * W8_PAD;
    uint32_t *sx = reinterpret_cast<uint32_t *>(reinterpret_cast<uint64_t *>(
                       reinterpret_cast<ulonglong2 *>(w8_smem) + W8_WARPS * W8_PAD) +
                                                W8_WARPS * W8_PAD) + w * W8_PAD;
    const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long fresh = 0, keyed = 0, full = 0;
    for (uint32_t g = warp0; g < nT; g += nwarps) {
        const Seg s = T[g];
        if (s.flags & SEG_KEYS)
            keyed += s.len;
        else
            fresh += s.len;
        const uint32_t P = next_pow2(s.len);
        {
            // All loads first (P <= 8 * 32), then the shared-memory stores.
            Key kk[8];
            uint32_t ii[8];
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const uint32_t e = lane + c * 32;
                kk[c] = key_max();
                ii[c] = IDX_MAX;
                if (e < s.len) load_elem(a, s, e, kk[c], ii[c]);
            }
#pragma unroll
            for (int c = 0; c < 8; ++c) {
                const uint32_t e = lane + c * 32;
                if (e < P) {
                    sk[pad(e)] = from_key(kk[c]);
                    sx[pad(e)] = ii[c];
                }
            }
        }
        __syncwarp();
        const uint32_t f = warp_diff_bit(sk, s.len, lane);
        bool packed = false;
        if (f < 128) {
            if (a.warp_merge) {
                if (P <= 64)
                    warp_run_packed<2, true>(sk, sv, 0, s.len, f, lane);
                else if (P <= 128)
                    warp_run_packed<4, true>(sk, sv, 0, s.len, f, lane);
                else
                    warp_run_packed<8, true>(sk, sv, 0, s.len, f, lane);
            } else {
                if (P <= 64)
                    warp_run_packed<2>(sk, sv, 0, s.len, f, lane);
                else if (P <= 128)
                    warp_run_packed<4>(sk, sv, 0, s.len, f, lane);
                else
                    warp_run_packed<8>(sk, sv, 0, s.len, f, lane);
            }
            __syncwarp();
            packed = __all_sync(0xffffffffu, window_pairs_ok_ind(sk, sv, s.len, lane, 32));
            if (!packed) {
                packed = __all_sync(0xffffffffu, window_runs_short(sv, s.len, lane, 32));
                if (packed) sort_window_runs(sk, sv, s.len, lane, 32);
            }
            if (!packed) {
                full += s.len;
                if (P <= 64)
                    warp_sort_run<2>(sk, sx, 0, lane);
                else if (P <= 128)
                    warp_sort_run<4>(sk, sx, 0, lane);
                else
                    warp_sort_run<8>(sk, sx, 0, lane);
            }
        }
        __syncwarp();
        if (packed)
            finish_segment<true>(a, s, sk, sx, sv, lane, 32, N, c);
        else
            finish_segment<false>(a, s, sk, sx, sv, lane, 32, N, c);
        __syncwarp();
    }
    if (lane == 0 && (fresh | keyed)) {
        atomicAdd(&c->warp8_fresh, fresh);
        atomicAdd(&c->warp8_keyed, keyed);
        if (full) atomicAdd(&c->full_sorted, full);
    }
}

// ---- segments of 257..SMALL_CAP strings: groups of threads -----------------
// A CTA of SMALL_THREADS threads is split into groups of GT threads (2, 4 or
// 8 warps); each group sorts one segment of up to GT * SMALL_ITEMS strings at a
// time and synchronises on its own named barrier.  Segments are bucketed by
// size so that every thread holds 5..8 strings: small segments do not leave
// warps idle at CTA-wide barriers, and one SM overlaps the loads and sorts of
// up to 12 segments.
constexpr int SMALL_PAD = SMALL_CAP + SMALL_CAP / 8;
constexpr size_t BLOCK_SMEM = SMALL_PAD * (sizeof(ulonglong2) + sizeof(uint32_t) + sizeof(uint64_t));
constexpr uint32_t BLOCK_RUN = 32 * SMALL_ITEMS;  // one warp's run of packed keys

// Barrier among the GT threads of group gi: named barrier 1 + gi (0 is
// __syncthreads).  Immediate ids, so that a CTA claims only the barriers it
// uses (at most 5) and the SM's barriers do not limit occupancy.
template <int GT>
__device__ __forceinline__ void group_sync(uint32_t gi) {
    constexpr int G = SMALL_THREADS / GT;
    if (G == 1 || gi == 0)
        asm volatile("bar.sync 1, %0;" ::"n"(GT) : "memory");
    else if (G == 2 || gi == 1)
        asm volatile("bar.sync 2, %0;" ::"n"(GT) : "memory");
    else if (gi == 2)
        asm volatile("bar.sync 3, %0;" ::"n"(GT) : "memory");
    else
        asm volatile("bar.sync 4, %0;" ::"n"(GT) : "memory");
}

// Full-comparator sort of the span (multiple of BLOCK_RUN) records at padded
// positions 0..span-1 by the GT threads of a group (thread t): warp runs, then
// pairwise merge-path merges.
template <int GT, bool PK = true>
__device__ __noinline__ void group_sort_full(ulonglong2 *sk, uint32_t *sx, uint32_t span,
                                             uint32_t t, uint32_t gi) {
    const uint32_t nruns = span / BLOCK_RUN;
    const uint32_t lane = t & 31, gw = t >> 5;
    if (gw < nruns) warp_sort_run<SMALL_ITEMS, PK>(sk, sx, gw * BLOCK_RUN, lane);
    group_sync<GT>(gi);
    for (uint32_t run = BLOCK_RUN; run < span; run <<= 1) {
        const uint32_t o = t * SMALL_ITEMS;
        Key ok[SMALL_ITEMS];
        uint32_t ox[SMALL_ITEMS];
        const bool active = o < span;
        if (active) {
            const uint32_t a0 = o & ~(2 * run - 1);  // run: a power of two
            const uint32_t b0 = a0 + run;
            const uint32_t la = min(run, span - a0);
            const uint32_t lb = b0 < span ? min(run, span - b0) : 0u;
            const uint32_t d = o - a0;
            uint32_t ia = merge_split<PK>(sk, sx, a0, la, b0, lb, d);
            uint32_t ib = d - ia;
#pragma unroll
            for (int i = 0; i < SMALL_ITEMS; ++i) {
                bool take_a = ib >= lb;
                Key ka, kb;
                uint32_t xa = 0, xb = 0;
                if (ia < la) {
                    ka = to_key(sk[kslot<PK>(a0 + ia)]);
                    xa = sx[kslot<PK>(a0 + ia)];
                }
                if (ib < lb) {
                    kb = to_key(sk[kslot<PK>(b0 + ib)]);
                    xb = sx[kslot<PK>(b0 + ib)];
                    if (ia < la) take_a = !pair_lt(kb, xb, ka, xa);
                }
                if (take_a) {
                    ok[i] = ka;
                    ox[i] = xa;
                    ++ia;
                } else {
                    ok[i] = kb;
                    ox[i] = xb;
                    ++ib;
                }
            }
        }
        group_sync<GT>(gi);
        if (active) {
#pragma unroll
            for (int i = 0; i < SMALL_ITEMS; ++i) {
                sk[kslot<PK>(o + i)] = from_key(ok[i]);
                sx[kslot<PK>(o + i)] = ox[i];
            }
        }
        group_sync<GT>(gi);
    }
}

// Pairwise merge-path merges of the sorted packed-key runs of BLOCK_RUN in
// sv[0..span) until one run is left; SMALL_ITEMS outputs per thread and pass.
template <int GT, typename V = uint64_t>
__device__ __forceinline__ void group_merge_passes64(V *sv, uint32_t span, uint32_t t,
                                                     uint32_t gi) {
    constexpr V VMAX = (V)~(V)0;
    for (uint32_t run = BLOCK_RUN; run < span; run <<= 1) {
        const uint32_t o = t * SMALL_ITEMS;
        V ov[SMALL_ITEMS];
        const bool active = o < span;
        if (active) {
            const uint32_t a0 = o & ~(2 * run - 1);  // run: a power of two
            const uint32_t b0 = a0 + run;
            const uint32_t la = min(run, span - a0);
            const uint32_t lb = b0 < span ? min(run, span - b0) : 0u;
            const uint32_t d = o - a0;
            uint32_t ia = merge_split64<V>(sv, a0, la, b0, lb, d);
            uint32_t ib = d - ia;
#pragma unroll
            for (int i = 0; i < SMALL_ITEMS; ++i) {
                const V va = ia < la ? sv[pad(a0 + ia)] : VMAX;
                const V vb = ib < lb ? sv[pad(b0 + ib)] : VMAX;
                const bool take_a = ib >= lb || (ia < la && va < vb);
                ov[i] = take_a ? va : vb;
                ia += take_a;
                ib += !take_a;
            }
        }
        group_sync<GT>(gi);
        if (active) {
#pragma unroll
            for (int i = 0; i < SMALL_ITEMS; ++i) sv[pad(o + i)] = ov[i];
        }
        group_sync<GT>(gi);
    }
}

// The CTAs cta0 .. cta0 + ncta - 1 of the launch sort the segments of one
// size class (list S of nS segments) with groups of GT threads.  LEAN: the
// finish takes neighbour LCPs from the packed windows (finish_packed).
// VAR 0: full-key finish; 1: LEAN; 2: LEAN, and the first sort is on 32-bit
// packed keys (half the work of the 64-bit network), widened to 64-bit keys
// afterwards; ties on their 21 window bits are then put in order in place.
template <int GT, int VAR = 0>
__device__ __forceinline__ void block_class(const SortArgs &a, const Seg *__restrict__ S,
                                            uint32_t nS, uint32_t cta0, uint32_t ncta, Seg *N,
                                            Counters *c) {
    constexpr uint32_t G = SMALL_THREADS / GT;          // groups per CTA
    constexpr uint32_t CAP = GT * SMALL_ITEMS;          // strings per group
    constexpr uint32_t PADC = CAP + CAP / 8;            // padded slots per group
    static_assert(G * PADC == SMALL_PAD, "group slots");
    extern __shared__ __align__(16) unsigned char block_smem[];
    __shared__ uint64_t red[2][SMALL_THREADS / 32];
    __shared__ int ok_flag[G], fix_flag[G], nar_flag[G];
    constexpr bool LEAN = VAR >= 1;
    const uint32_t gi = threadIdx.x / GT, t = threadIdx.x % GT;
    const uint32_t lane = threadIdx.x & 31, gw = t >> 5, w = threadIdx.x >> 5;
    ulonglong2 *sk_all = reinterpret_cast<ulonglong2 *>(block_smem);
    uint64_t *sv_all = reinterpret_cast<uint64_t *>(sk_all + SMALL_PAD);
    uint32_t *sx_all = reinterpret_cast<uint32_t *>(sv_all + SMALL_PAD);
    ulonglong2 *sk = sk_all + gi * PADC;
    uint64_t *sv = sv_all + gi * PADC;
    uint32_t *sx = sx_all + gi * PADC;
    unsigned long long fresh = 0, keyed = 0, full = 0;
    for (uint32_t g = (blockIdx.x - cta0) * G + gi; g < nS; g += ncta * G) {
        const Seg s = S[g];
        if (s.flags & SEG_KEYS)
            keyed += s.len;
        else
            fresh += s.len;
        const uint32_t nruns = (s.len + BLOCK_RUN - 1) / BLOCK_RUN;
        const uint32_t span = nruns * BLOCK_RUN;
        {
            // All of a thread's loads first (span <= SMALL_ITEMS * GT), so
            // that they are in flight together, then the shared-memory stores.
            Key kk[SMALL_ITEMS];
            uint32_t ii[SMALL_ITEMS];
#pragma unroll
            for (int c = 0; c < SMALL_ITEMS; ++c) {
                const uint32_t e = t + c * GT;
                kk[c] = key_max();
                ii[c] = IDX_MAX;
                if (e < s.len) load_elem(a, s, e, kk[c], ii[c]);
            }
#pragma unroll
            for (int c = 0; c < SMALL_ITEMS; ++c) {
                const uint32_t e = t + c * GT;
                if (e < span) {
                    sk[pad(e)] = from_key(kk[c]);
                    sx[pad(e)] = ii[c];
                }
            }
        }
        if (t == 0) ok_flag[gi] = fix_flag[gi] = nar_flag[gi] = 1;
        group_sync<GT>(gi);
        // f: first bit in which the keys differ.
        {
            const Key k0 = to_key(sk[pad(0)]);
            uint64_t dh = 0, dl = 0;
            for (uint32_t e = t; e < s.len; e += GT) {
                const Key k = to_key(sk[pad(e)]);
                dh |= k.hi ^ k0.hi;
                dl |= k.lo ^ k0.lo;
            }
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                dh |= __shfl_xor_sync(0xffffffffu, dh, d);
                dl |= __shfl_xor_sync(0xffffffffu, dl, d);
            }
            if (lane == 0) {
                red[0][w] = dh;
                red[1][w] = dl;
            }
        }
        group_sync<GT>(gi);
        uint64_t dh = 0, dl = 0;
#pragma unroll
        for (uint32_t q = 0; q < GT / 32; ++q) {
            dh |= red[0][gi * (GT / 32) + q];
            dl |= red[1][gi * (GT / 32) + q];
        }
        bool packed = false;
        const uint32_t f = (dh | dl) ? clz128(dh, dl) : 128u;
        if (f < 128) {
            bool sorted64 = false;
            if constexpr (VAR == 2) {
                uint32_t *sv32 = reinterpret_cast<uint32_t *>(sv);  // same bytes
                if (gw < nruns)
                    warp_run_packed32<SMALL_ITEMS>(sk, sv32, gw * BLOCK_RUN, s.len, f, lane);
                group_sync<GT>(gi);
                group_merge_passes64<GT, uint32_t>(sv32, span, t, gi);
                // Widen to 64-bit packed keys in this order; the two arrays
                // share their bytes, so the values pass through registers.
                const uint32_t o = t * SMALL_ITEMS;
                uint32_t pv[SMALL_ITEMS];
#pragma unroll
                for (int i = 0; i < SMALL_ITEMS; ++i)
                    pv[i] = o + i < span ? sv32[pad(o + i)] : 0u;
                group_sync<GT>(gi);
#pragma unroll
                for (int i = 0; i < SMALL_ITEMS; ++i) {
                    const uint32_t e = o + i;
                    if (e < s.len) {
                        const uint32_t pos = pv[i] & (uint32_t)POS_MASK;
                        sv[pad(e)] = sort_key(to_key(sk[pad(pos)]), f, pos);
                    }
                }
                group_sync<GT>(gi);
                if (!sort_narrow_runs(sv, s.len, t, GT)) nar_flag[gi] = 0;
                group_sync<GT>(gi);
                sorted64 = nar_flag[gi] != 0;
            }
            if (!sorted64) {
                if (gw < nruns) {
                    if (a.warp_merge)
                        warp_run_packed<SMALL_ITEMS, true>(sk, sv, gw * BLOCK_RUN, s.len, f, lane);
                    else
                        warp_run_packed<SMALL_ITEMS>(sk, sv, gw * BLOCK_RUN, s.len, f, lane);
                }
                group_sync<GT>(gi);
                group_merge_passes64<GT>(sv, span, t, gi);
            }
            if (!window_pairs_ok_ind(sk, sv, s.len, t, GT)) ok_flag[gi] = 0;
            group_sync<GT>(gi);
            packed = ok_flag[gi] != 0;
            if (!packed) {
                if (!window_runs_short(sv, s.len, t, GT)) fix_flag[gi] = 0;
                group_sync<GT>(gi);
                packed = fix_flag[gi] != 0;
                if (packed) {
                    sort_window_runs(sk, sv, s.len, t, GT);
                } else {
                    if (t == 0) full += s.len;
                    group_sort_full<GT>(sk, sx, span, t, gi);
                }
            }
        }
        group_sync<GT>(gi);
        if (packed && LEAN)
            finish_packed<true>(a, s, sk, sx, sv, f, t, GT, N, c);
        else if (packed)
            finish_segment<true>(a, s, sk, sx, sv, t, GT, N, c);
        else
            finish_segment<false>(a, s, sk, sx, sv, t, GT, N, c);
        group_sync<GT>(gi);
    }
    if (t == 0 && (fresh | keyed)) {
        atomicAdd(&c->block_fresh, fresh);
        atomicAdd(&c->block_keyed, keyed);
        if (full) atomicAdd(&c->full_sorted, full);
    }
}

// One size class per launch (a single launch for all three inlines all
// three bodies and spills more; measured slower).
template <int GT, int VAR>
__global__ void __launch_bounds__(SMALL_THREADS, 3) k_block(SortArgs a, const Seg *__restrict__ S,
                                                            Span sp, Seg *N, Counters *c) {
    const uint32_t lo = count_of(sp.lo);
    block_class<GT, VAR>(a, S + lo, count_of(sp.hi) - lo, 0, gridDim.x, N, c);
}

// ---- segments of 257..SMALL_CAP strings, with the next segment prefetched ---
// The same thread groups and sort as k_block, but a group's records (16-byte
// key, index) of a keyed segment reach shared memory through cp.async (global
// -> shared copies that bypass the registers), issued for the group's NEXT
// segment before it sorts the current one, so that the copy runs under the
// sort.  Two record buffers per group (contiguous slots: the copies cannot
// write the padded layout); the packed keys are built from the records
// loaded once into registers.  Segments without keys at their depth (fresh)
// are gathered by the group's threads as in k_block.
constexpr size_t BLOCK2_SMEM =
    2 * (size_t)SMALL_CAP * (sizeof(ulonglong2) + sizeof(uint32_t)) + SMALL_PAD * sizeof(uint64_t);

__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void *smem, const void *gmem) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
// Waits until at most N of this thread's committed copy groups are pending.
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

template <int GT>
__device__ __forceinline__ void block2_class(const SortArgs &a, const Seg *__restrict__ S,
                                             uint32_t nS, Seg *N, Counters *c) {
    constexpr uint32_t G = SMALL_THREADS / GT;  // groups per CTA
    constexpr uint32_t CAP = GT * SMALL_ITEMS;  // strings per group
    constexpr uint32_t PADC = CAP + CAP / 8;    // padded packed-key slots per group
    static_assert(G * PADC == SMALL_PAD, "group slots");
    extern __shared__ __align__(16) unsigned char block_smem[];
    __shared__ uint64_t red[2][SMALL_THREADS / 32];
    __shared__ int ok_flag[G], fix_flag[G];
    const uint32_t gi = threadIdx.x / GT, t = threadIdx.x % GT;
    const uint32_t lane = threadIdx.x & 31, gw = t >> 5, w = threadIdx.x >> 5;
    ulonglong2 *rk_all = reinterpret_cast<ulonglong2 *>(block_smem);  // [2][SMALL_CAP]
    uint32_t *rx_all = reinterpret_cast<uint32_t *>(rk_all + 2 * SMALL_CAP);
    uint64_t *sv = reinterpret_cast<uint64_t *>(rx_all + 2 * SMALL_CAP) + gi * PADC;
    unsigned long long fresh = 0, keyed = 0, full = 0;
    const uint32_t stride = gridDim.x * G;
    // Copies of a keyed segment's records into record buffer `buf`; every
    // thread commits one copy group per call (empty when there is nothing).
    auto prefetch = [&](const Seg &q, uint32_t buf) {
        if (q.len && (q.flags & SEG_KEYS)) {
            const int b = q.flags & SEG_BUF1;
            const ulonglong2 *K = a.keyb(b) + q.start;
            const uint32_t *I = a.idxb(b) + q.start;
            ulonglong2 *dk = rk_all + buf * SMALL_CAP + gi * CAP;
            uint32_t *dx = rx_all + buf * SMALL_CAP + gi * CAP;
#pragma unroll
            for (int cc = 0; cc < SMALL_ITEMS; ++cc) {
                const uint32_t e = t + cc * GT;
                if (e < q.len) {
                    cp_async16(dk + e, K + e);
                    cp_async4(dx + e, I + e);
                }
            }
        }
        cp_async_commit();
    };
    const Seg none{0, 0, 0, 0};
    uint32_t g = blockIdx.x * G + gi;
    Seg s_cur = g < nS ? S[g] : none;
    Seg s_nxt = g + stride < nS ? S[g + stride] : none;
    prefetch(s_cur, 0);
    uint32_t cb = 0;
    for (; g < nS; g += stride, cb ^= 1) {
        const Seg s = s_cur;
        prefetch(s_nxt, cb ^ 1);
        s_cur = s_nxt;
        s_nxt = g + 2 * stride < nS ? S[g + 2 * stride] : none;
        ulonglong2 *sk = rk_all + cb * SMALL_CAP + gi * CAP;
        uint32_t *sx = rx_all + cb * SMALL_CAP + gi * CAP;
        if (s.flags & SEG_KEYS) {
            keyed += s.len;
        } else {
            fresh += s.len;
            // Gather at this depth: all of a thread's loads first.
            Key kk[SMALL_ITEMS];
            uint32_t ii[SMALL_ITEMS];
#pragma unroll
            for (int cc = 0; cc < SMALL_ITEMS; ++cc) {
                const uint32_t e = t + cc * GT;
                if (e < s.len) load_elem(a, s, e, kk[cc], ii[cc]);
            }
#pragma unroll
            for (int cc = 0; cc < SMALL_ITEMS; ++cc) {
                const uint32_t e = t + cc * GT;
                if (e < s.len) {
                    sk[e] = from_key(kk[cc]);
                    sx[e] = ii[cc];
                }
            }
        }
        cp_async_wait<1>();  // this segment's copies (the next one's may run on)
        if (t == 0) ok_flag[gi] = fix_flag[gi] = 1;
        group_sync<GT>(gi);
        // f: first bit in which the keys differ (thread t's records are
        // t, t + GT, ...; contiguous across threads, so no bank conflicts).
        {
            const Key k0 = to_key(sk[0]);
            uint64_t dh = 0, dl = 0;
#pragma unroll
            for (int cc = 0; cc < SMALL_ITEMS; ++cc) {
                const uint32_t e = t + cc * GT;
                if (e < s.len) {
                    const Key k = to_key(sk[e]);
                    dh |= k.hi ^ k0.hi;
                    dl |= k.lo ^ k0.lo;
                }
            }
#pragma unroll
            for (int d = 16; d > 0; d >>= 1) {
                dh |= __shfl_xor_sync(0xffffffffu, dh, d);
                dl |= __shfl_xor_sync(0xffffffffu, dl, d);
            }
            if (lane == 0) {
                red[0][w] = dh;
                red[1][w] = dl;
            }
        }
        group_sync<GT>(gi);
        uint64_t dh = 0, dl = 0;
#pragma unroll
        for (uint32_t q = 0; q < GT / 32; ++q) {
            dh |= red[0][gi * (GT / 32) + q];
            dl |= red[1][gi * (GT / 32) + q];
        }
        bool packed = false;
        const uint32_t f = (dh | dl) ? clz128(dh, dl) : 128u;
        if (f < 128) {
            // Every warp of the group sorts the packed keys of its own
            // records (t, t + GT, ...; any split of the records works: the
            // position in the low bits identifies each one); positions past
            // the end pad as distinct values above every real one.
            uint64_t v[SMALL_ITEMS];
#pragma unroll
            for (int cc = 0; cc < SMALL_ITEMS; ++cc) {
                const uint32_t e = t + cc * GT;
                v[cc] = e < s.len ? sort_key(to_key(sk[e]), f, e) : ((~0ull << POS_BITS) | e);
            }
            warp_bitonic64<SMALL_ITEMS>(v, lane);
#pragma unroll
            for (int i = 0; i < SMALL_ITEMS; ++i) sv[pad(gw * BLOCK_RUN + lane * SMALL_ITEMS + i)] = v[i];
            group_sync<GT>(gi);
            group_merge_passes64<GT>(sv, CAP, t, gi);
            if (!window_pairs_ok_ind<false>(sk, sv, s.len, t, GT)) ok_flag[gi] = 0;
            group_sync<GT>(gi);
            packed = ok_flag[gi] != 0;
            if (!packed) {
                if (!window_runs_short(sv, s.len, t, GT)) fix_flag[gi] = 0;
                group_sync<GT>(gi);
                packed = fix_flag[gi] != 0;
                if (packed) {
                    sort_window_runs<false>(sk, sv, s.len, t, GT);
                } else {
                    // Full comparator over the whole group span (rare): the
                    // slots past the end sort last.
                    for (uint32_t e = s.len + t; e < CAP; e += GT) {
                        sk[e] = from_key(key_max());
                        sx[e] = IDX_MAX;
                    }
                    group_sync<GT>(gi);
                    if (t == 0) full += s.len;
                    group_sort_full<GT, false>(sk, sx, CAP, t, gi);
                }
            }
        }
        group_sync<GT>(gi);
        if (packed)
            finish_packed<false>(a, s, sk, sx, sv, f, t, GT, N, c);
        else
            finish_segment<false, false>(a, s, sk, sx, sv, t, GT, N, c);
        group_sync<GT>(gi);
    }
    cp_async_wait<0>();
    if (t == 0 && (fresh | keyed)) {
        atomicAdd(&c->block_fresh, fresh);
        atomicAdd(&c->block_keyed, keyed);
        if (full) atomicAdd(&c->full_sorted, full);
    }
}

template <int GT>
__global__ void __launch_bounds__(SMALL_THREADS, 2) k_block2(SortArgs a, const Seg *__restrict__ S,
                                                             Span sp, Seg *N, Counters *c) {
    const uint32_t lo = count_of(sp.lo);
    block2_class<GT>(a, S + lo, count_of(sp.hi) - lo, N, c);
}

// ---- equality buckets: work items of up to EQ_TILE strings ------------------
__global__ void k_equal(SortArgs a, const Seg *__restrict__ E0, Span sp, Seg *N, Counters *c) {
    const uint32_t lo = count_of(sp.lo);
    const Seg *__restrict__ E = E0 + lo;
    const uint32_t nE = count_of(sp.hi) - lo;
    unsigned long long moved = 0, fin = 0;
    for (uint32_t g = blockIdx.x; g < nE; g += gridDim.x) {
        const Seg s = E[g];
        const int b = s.flags & SEG_BUF1;
        const uint32_t ch = s.flags >> SEG_CHUNK_SHIFT;
        const Key k = to_key(a.keyb(b)[s.start]);
        const bool end = key_is_end(k);
        if (ch == 0 && threadIdx.x == 0) {
            a.key[0][s.start] = from_key(k);
            a.key[0][s.start + s.len - 1] = from_key(k);
            if (!end) emit_next(N, c, s.start, s.len, s.depth + KEY_BYTES);
        }
        const uint32_t lo = ch * EQ_TILE;
        const uint32_t hi = min(lo + (uint32_t)EQ_TILE, s.len);
        if (threadIdx.x == 0) {
            if (b) moved += hi - lo;
            if (end) fin += hi - lo;
        }
        const uint32_t l = s.depth + key_len(k);
        for (uint32_t i = lo + threadIdx.x; i < hi; i += blockDim.x) {
            const uint32_t p = s.start + i;
            if (b) a.idx[0][p] = a.idx[1][p];
            if (end && i > 0) a.lcp[p] = l;
        }
    }
    if (threadIdx.x == 0 && (moved | fin)) {
        atomicAdd(&c->equal_moved, moved);
        atomicAdd(&c->equal_final, fin);
    }
}

__global__ void k_boundary(SortArgs a, const uint2 *__restrict__ B, Counters *c) {
    const uint32_t nB = c->n_bound;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nB; i += gridDim.x * blockDim.x) {
        const uint2 e = B[i];
        a.lcp[e.x] = e.y + key_lcp(to_key(a.key[0][e.x - 1]), to_key(a.key[0][e.x]));
    }
}

// ---- control kernels of the device-driven round loop --------------------------
// The graph's loops (rounds, partition levels) and branches (separate gather,
// gathering count) are CUDA graph conditional nodes; these kernels read the
// device counters and set their conditions, so no host round trip is needed
// between launches.  None of them waits on another block: the multi-CTA ones
// copy a list and let the last CTA to finish (atomic ticket) do the update.

// Each loop body first clears its own condition, and only the kernel that
// ends the body sets it again when another iteration is due: a body whose
// last kernel did not run cannot repeat.
__global__ void k_g_round_begin(GraphState *g, Counters *c, cudaGraphConditionalHandle h_round) {
    uint32_t *w = reinterpret_cast<uint32_t *>(c);
    for (uint32_t i = threadIdx.x; i < sizeof(Counters) / 4; i += blockDim.x) w[i] = 0;
    if (threadIdx.x == 0) {
        cudaGraphSetConditional(h_round, 0u);
        g->cur_w1 = g->cur_w8 = g->cur_e = 0;
        g->cur_s[0] = g->cur_s[1] = g->cur_s[2] = 0;
        g->levels = 0;
    }
}

__global__ void k_g_after_classify(GraphState *g, const Counters *c,
                                   cudaGraphConditionalHandle h_level,
                                   cudaGraphConditionalHandle h_gather) {
    if (threadIdx.x != 0) return;
    const uint32_t nl = c->n_large;
    g->n_large = nl;
    g->levels = 0;
    if (g->round < 64) g->live[g->round] = c->live_next;
    const bool fused = gather_fused(g->fused, g->round == 0, c->gather_elems);
    g->fused_round = fused ? 1u : 0u;
    g->first = fused ? 1u : 0u;
    cudaGraphSetConditional(h_gather, (nl > 0 && !fused) ? 1u : 0u);
    cudaGraphSetConditional(h_level, nl > 0 ? 1u : 0u);
}

__global__ void k_g_level_begin(const GraphState *g, cudaGraphConditionalHandle h_level,
                                cudaGraphConditionalHandle h_first) {
    if (threadIdx.x != 0) return;
    cudaGraphSetConditional(h_level, 0u);
    cudaGraphSetConditional(h_first, g->first ? 1u : 0u);
}

// True in thread 0 of the last CTA of the grid to get here (after its own
// writes are visible); that CTA resets the ticket for the next launch.
__device__ __forceinline__ bool last_cta(uint32_t *ticket) {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last || threadIdx.x != 0) return false;
    __threadfence();
    *ticket = 0;
    return true;
}

__global__ void k_g_level_end(GraphState *g, Counters *c, Seg *L, const Seg *__restrict__ L2,
                              cudaGraphConditionalHandle h_level) {
    const uint32_t n = c->n_large_next;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        L[i] = L2[i];
    if (!last_cta(&g->ticket)) return;
    g->n_large = n;
    c->n_large_next = 0;
    g->first = 0;
    g->levels += 1;
    g->partition_levels += 1;
    g->cur_w1 = c->n_w1;
    g->cur_w8 = c->n_w8;
    g->cur_s[0] = c->n_small;
    g->cur_s[1] = c->n_small2;
    g->cur_s[2] = c->n_small3;
    g->cur_e = c->n_equal;
    bool more = n > 0;
    if (more && g->levels >= g->max_levels) {
        g->error = 1;  // reported by the host as an internal error, not a hang
        more = false;
    }
    cudaGraphSetConditional(h_level, more ? 1u : 0u);
}

__global__ void k_g_round_end(GraphState *g, const Counters *c, Seg *R, const Seg *__restrict__ N,
                              cudaGraphConditionalHandle h_round) {
    const uint32_t n = c->n_next;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        R[i] = N[i];
    if (!last_cta(&g->ticket)) return;
    const bool fused = g->fused_round != 0;
    g->small_segments += (unsigned long long)c->n_w1 + c->n_w8 + c->n_small + c->n_small2 +
                         c->n_small3;
    g->partitioned += c->partitioned;
    g->gather_elems += c->gather_elems;
    if (fused) g->gather_fused += c->gather_elems;
    g->warp1_fresh += c->warp1_fresh;
    g->warp1_keyed += c->warp1_keyed;
    g->warp8_fresh += c->warp8_fresh;
    g->warp8_keyed += c->warp8_keyed;
    g->block_fresh += c->block_fresh;
    g->block_keyed += c->block_keyed;
    g->equal_moved += c->equal_moved;
    g->equal_final += c->equal_final;
    g->boundaries += c->n_bound;
    g->warp1_deep += c->warp1_deep;
    g->full_sorted += c->full_sorted;
    g->window_saved += c->window_saved;
    g->window_used += c->window_used;
    if (c->error) g->error = 2;  // a scan's look-back waited past its bound
    g->n_cur = n;
    g->round += 1;
    g->round_in_launch += 1;
    g->done = n == 0 ? 1u : 0u;
    const bool more = n > 0 && !g->error && g->round_in_launch < GRAPH_ROUNDS_PER_LAUNCH;
    cudaGraphSetConditional(h_round, more ? 1u : 0u);
}

// ---- exclusive scan (u32), one pass with decoupled look-back ---------------
// Each CTA takes the next tile from a ticket (so every tile it waits for has
// started), scans its 4096 values, publishes its sum, and warp 0 walks back
// over its predecessors' status words 32 at a time, adding sums until it
// meets an inclusive prefix; then it publishes its own inclusive prefix.
// Status word: flag (1 = tile sum, 2 = inclusive prefix) << 32 | value.  The
// wait for a predecessor is bounded; past the bound the CTA records an
// error and goes on (the host reports it; the result is then not used).
constexpr uint64_t LB_SUM = 1ull << 32, LB_INCL = 2ull << 32;
constexpr uint32_t LB_SPIN_MAX = 1u << 22;

__device__ __forceinline__ uint32_t warp_sum32(uint32_t v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v += __shfl_xor_sync(0xffffffffu, v, d);
    return v;
}

__global__ void __launch_bounds__(SCAN_THREADS) k_scan_lookback(const uint32_t *in, uint32_t *out,
                                                                Count cnt,
                                                                unsigned long long *status,
                                                                uint32_t *ticket, uint32_t *err) {
    __shared__ uint32_t buf[SCAN_CHUNK];
    __shared__ uint32_t s_tile, s_prefix;
    const uint32_t n = count_of(cnt);
    const uint32_t lane = threadIdx.x & 31;
    if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
    __syncthreads();
    const uint32_t t = s_tile;
    const uint64_t base = (uint64_t)t * SCAN_CHUNK;
    if (base >= n) {
        if (n == 0 && t == 0 && threadIdx.x == 0) out[0] = 0;
        return;
    }
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const int j = k * SCAN_THREADS + threadIdx.x;
        const uint64_t i = base + j;
        buf[j] = i < n ? in[i] : 0;
    }
    __syncthreads();
    uint32_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) s += buf[threadIdx.x * SCAN_ITEMS + k];
    uint32_t excl;
    const uint32_t total = block_exclusive_scan(s, excl);
    if (threadIdx.x < 32) {
        uint32_t prefix = 0;
        if (t == 0) {
            if (lane == 0) atomicExch(&status[0], LB_INCL | total);
        } else {
            if (lane == 0) atomicExch(&status[t], LB_SUM | total);
            int64_t j = (int64_t)t - 1;  // nearest predecessor not yet added
            uint32_t spins = 0;
            bool failed = false;
            while (true) {
                const int64_t idx = j - (int64_t)lane;
                const volatile unsigned long long *sp = status + (idx >= 0 ? idx : 0);
                unsigned long long w = idx >= 0 ? *sp : LB_INCL;
                while (__any_sync(0xffffffffu, (w >> 32) == 0)) {
                    if (++spins > LB_SPIN_MAX) {
                        failed = true;
                        break;
                    }
                    __nanosleep(32);
                    if ((w >> 32) == 0) w = *sp;
                }
                if (failed) break;
                const uint32_t incl = __ballot_sync(0xffffffffu, (w >> 32) == 2);
                if (incl) {
                    const uint32_t k = __ffs(incl) - 1;  // the nearest inclusive prefix
                    prefix += warp_sum32(lane <= k ? (uint32_t)w : 0u);
                    break;
                }
                prefix += warp_sum32((uint32_t)w);
                j -= 32;
            }
            if (lane == 0) {
                if (failed) atomicExch(err, 1u);
                atomicExch(&status[t], LB_INCL | (prefix + total));
            }
        }
        if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();
    uint32_t run = s_prefix + excl;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const int j = threadIdx.x * SCAN_ITEMS + k;
        const uint32_t v = buf[j];
        buf[j] = run;
        run += v;
    }
    __syncthreads();
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const int j = k * SCAN_THREADS + threadIdx.x;
        const uint64_t i = base + j;
        if (i < n) out[i] = buf[j];
    }
    if (threadIdx.x == 0 && base + SCAN_CHUNK >= n) out[n] = s_prefix + total;
}

}  // namespace

// ---- launchers --------------------------------------------------------------
static inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

// Opt-in to more than 48 KB of dynamic shared memory for the kernels that use
// it.  The attribute belongs to the function in the current device's context,
// so it is set once per device (bit d of the mask), for all kernels at once;
// two threads that race here both set the same values, which is harmless.
static constexpr int SAMPLE_SMEM =
    (SAMPLES_MAX + SAMPLES_MAX / 8) * sizeof(uint64_t) + SAMPLE_KEEP * sizeof(ulonglong2);
static void set_smem_attrs() {
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0) return;  // the launch reports it
    const uint64_t bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return;
    cudaFuncSetAttribute(k_sample, cudaFuncAttributeMaxDynamicSharedMemorySize, SAMPLE_SMEM);
    cudaFuncSetAttribute(k_count<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(PartSmem));
    cudaFuncSetAttribute(k_count<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(PartSmem));
    cudaFuncSetAttribute(k_scatter<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(ScatterSmem));
    cudaFuncSetAttribute(k_scatter<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(ScatterSmem));
    cudaFuncSetAttribute(k_scatter2, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)sizeof(Scatter2Smem));
    cudaFuncSetAttribute(k_warp8, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)W8_SMEM);
    cudaFuncSetAttribute(k_block<64, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<64, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<64, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<128, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<128, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<128, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<256, 0>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<256, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block<256, 2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK_SMEM);
    cudaFuncSetAttribute(k_block2<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK2_SMEM);
    cudaFuncSetAttribute(k_block2<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK2_SMEM);
    cudaFuncSetAttribute(k_block2<256>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         (int)BLOCK2_SMEM);
    done.fetch_or(bit, std::memory_order_release);
}

void launch_iota(uint32_t *idx, uint32_t n, cudaStream_t st) {
    const uint32_t g = cdiv(n, 256) < 148 * 16 ? cdiv(n, 256) : 148 * 16;
    k_iota<<<g ? g : 1, 256, 0, st>>>(idx, n);
}

// Grid for a launcher given `grid` (> 0: as given) or a host count of work
// units of `per` each (capped at cap CTAs; 0 when there is no work).
static int grid_of(int grid, const Count &n, uint32_t per, uint32_t cap) {
    if (grid > 0) return grid;
    if (n.dev) return (int)cap;
    const uint32_t g = cdiv(n.host, per);
    return (int)(g < cap ? g : cap);
}

void launch_classify(const Seg *R, Count nR, uint32_t warp8_cap, Seg *W1, Seg *W8,
                     SmallLists S, Seg *L, Counters *c, int grid, cudaStream_t st) {
    const int g = grid_of(grid, nR, 256, 1u << 30);
    if (!g) return;
    k_classify<<<g, 256, 0, st>>>(R, nR, warp8_cap, W1, W8, S, L, c);
}

void launch_init_batch(const uint32_t *inst_start, uint32_t ninst, Seg *R, uint32_t *lcp,
                       Counters *c, cudaStream_t st) {
    if (!ninst) return;
    k_init_batch<<<cdiv(ninst, 256), 256, 0, st>>>(inst_start, ninst, R, lcp, c);
}

void launch_localize(uint32_t *perm, uint32_t n, const uint32_t *inst_start, uint32_t ninst,
                     cudaStream_t st) {
    const uint32_t g = cdiv(n, 256) < 148 * 8 ? cdiv(n, 256) : 148 * 8;
    k_localize<<<g ? g : 1, 256, 0, st>>>(perm, n, inst_start, ninst);
}

void launch_join(uint64_t *goffs, uint32_t *lcp, uint32_t *perm, const ReqJob *jobs,
                 uint32_t njobs, uint32_t total, Seg *R, cudaStream_t st) {
    if (!njobs || !total) return;
    const uint32_t g = cdiv(total, 256) < 148 * 8 ? cdiv(total, 256) : 148 * 8;
    k_join<<<g, 256, 0, st>>>(goffs, lcp, perm, jobs, njobs, total, R);
}

void launch_mark(const Seg *R, uint32_t nR, const uint32_t *base, uint32_t nact, uint32_t *flag,
                 cudaStream_t st) {
    if (!nR || !nact) return;
    const uint32_t g = cdiv(nR, 256) < 148 * 8 ? cdiv(nR, 256) : 148 * 8;
    k_mark<<<g, 256, 0, st>>>(R, nR, base, nact, flag);
}

void launch_unbase(uint32_t *perm, const ReqJob *jobs, uint32_t njobs, uint32_t total,
                   cudaStream_t st) {
    if (!njobs || !total) return;
    const uint32_t g = cdiv(total, 256) < 148 * 8 ? cdiv(total, 256) : 148 * 8;
    k_unbase<<<g, 256, 0, st>>>(perm, jobs, njobs, total);
}

uint64_t text_tiles(uint64_t len) { return (len + TEXT_TILE - 1) / TEXT_TILE; }

void launch_text_count(const uint8_t *text, uint64_t len, uint8_t delim, uint32_t *tile_cnt,
                       unsigned long long *total, cudaStream_t st) {
    const uint64_t t = text_tiles(len);
    if (t) k_text_count<<<(unsigned)t, TEXT_THREADS, 0, st>>>(text, len, delim, tile_cnt, total);
}

void launch_text_starts(uint8_t *text, uint64_t len, uint8_t delim, const uint32_t *tile_base,
                        uint64_t n, void *offs, int off_width, cudaStream_t st) {
    const uint64_t t = text_tiles(len);
    if (t)
        k_text_starts<<<(unsigned)t, TEXT_THREADS, 0, st>>>(text, len, delim, tile_base, n, offs,
                                                            off_width);
}

void launch_iota_offs(void *offs, int off_width, uint64_t n, cudaStream_t st) {
    const uint64_t g = (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16;
    k_iota_offs<<<(unsigned)(g ? g : 1), 256, 0, st>>>(offs, off_width, n);
}

void launch_sorted_offs(const uint32_t *perm, const void *offs, int off_width, uint64_t n,
                        void *out, int out_width, cudaStream_t st) {
    const uint64_t g = (n + 255) / 256 < 148 * 16 ? (n + 255) / 256 : 148 * 16;
    k_sorted_offs<<<(unsigned)(g ? g : 1), 256, 0, st>>>(perm, offs, off_width, n, out,
                                                         out_width);
}

void launch_byte_hist(const uint8_t *arena, uint64_t arena_bytes, const void *offs, int off_width,
                      uint32_t n, uint32_t samples, uint32_t *hist, cudaStream_t st) {
    k_byte_hist<<<1, 256, 0, st>>>(arena, arena_bytes, offs, off_width, n, samples, hist);
}

void launch_scan_pair(const uint32_t *in0, uint32_t *out0, const uint32_t *in1, uint32_t *out1,
                      Count n, cudaStream_t st) {
    k_scan_pair<<<1, SMALL_SCAN_THREADS, 0, st>>>(in0, out0, in1, out1, n);
}

void launch_seg_tiles(const Seg *segs, Count n, uint32_t tile, uint32_t *out, cudaStream_t st) {
    k_seg_tiles<<<1, SMALL_SCAN_THREADS, 0, st>>>(segs, n, tile, out);
}

uint32_t scan_partials_needed(uint32_t n) { return cdiv(n ? n : 1, SCAN_CHUNK) + 1; }

size_t lookback_state_bytes(uint32_t cap) { return 8 + (size_t)cdiv(cap ? cap : 1, SCAN_CHUNK) * 8; }

void launch_scan_lookback(const uint32_t *in, uint32_t *out, uint32_t cap, Count n,
                          unsigned char *state, uint32_t *err, cudaStream_t st) {
    const uint32_t nb = cdiv(cap ? cap : 1, SCAN_CHUNK);
    k_scan_lookback<<<nb, SCAN_THREADS, 0, st>>>(in, out, n,
                                                  reinterpret_cast<unsigned long long *>(state + 8),
                                                  reinterpret_cast<uint32_t *>(state), err);
}

void launch_scan(const uint32_t *in, uint32_t *out, uint32_t cap, Count n, uint32_t *partials,
                 cudaStream_t st) {
    const uint32_t nb = cdiv(cap ? cap : 1, SCAN_CHUNK);
    k_scan_reduce<<<nb, SCAN_THREADS, 0, st>>>(in, n, partials);
    k_scan_partials<<<1, SCAN_THREADS, 0, st>>>(partials, nb);
    k_scan_down<<<nb, SCAN_THREADS, 0, st>>>(in, out, n, partials, nb);
}

void launch_gather(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                   Counters *c, int grid, cudaStream_t st) {
    if (!nL.dev && !nL.host) return;
    k_gather<<<grid, GATHER_THREADS, 0, st>>>(a, L, nL, tile_base, c);
}

void launch_sample(const SortArgs &a, const Seg *L, Count nL, ulonglong2 *spl, uint32_t *nspl,
                   uint16_t *tbl, uint32_t *ntiles, uint32_t *cm_size, bool from_arena, int grid,
                   cudaStream_t st) {
    const int g = grid_of(grid, nL, 1, 1u << 30);
    if (!g) return;
    set_smem_attrs();
    k_sample<<<g, SAMPLE_THREADS, SAMPLE_SMEM, st>>>(a, L, nL, spl, nspl, tbl, ntiles, cm_size,
                                                     from_arena);
}

void launch_count(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                  const ulonglong2 *spl, const uint32_t *nspl, const uint16_t *tbl,
                  const uint32_t *cm_base, uint32_t *cm, Counters *c, bool gather, int grid,
                  cudaStream_t st) {
    if (!nL.dev && !nL.host) return;
    set_smem_attrs();
    if (gather)
        k_count<true><<<grid, PART_THREADS, sizeof(PartSmem), st>>>(a, L, nL, tile_base, spl, nspl,
                                                                    tbl, cm_base, cm, c);
    else
        k_count<false><<<grid, PART_THREADS, sizeof(PartSmem), st>>>(a, L, nL, tile_base, spl,
                                                                     nspl, tbl, cm_base, cm, c);
}

void launch_scatter(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                    const ulonglong2 *spl, const uint32_t *nspl, const uint16_t *tbl,
                    const uint32_t *cm_base, const uint32_t *cm_scan, int grid, cudaStream_t st) {
    if (!nL.dev && !nL.host) return;
    set_smem_attrs();
    if (a.scatter_staged_idx == 2) {
        k_scatter<true><<<grid, SCATTER_THREADS, sizeof(ScatterSmem), st>>>(
            a, L, nL, tile_base, nspl, cm_base, cm_scan);
        return;
    }
    if (a.scatter_staged_idx) {
        // three CTAs per SM where k_scatter fits two (grid: two per SM)
        k_scatter2<<<grid / 2 * 3, SCATTER_THREADS, sizeof(Scatter2Smem), st>>>(
            a, L, nL, tile_base, nspl, cm_base, cm_scan);
        return;
    }
    k_scatter<false><<<grid, SCATTER_THREADS, sizeof(ScatterSmem), st>>>(
        a, L, nL, tile_base, nspl, cm_base, cm_scan);
}

void launch_emit(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                 const uint32_t *nspl, const uint32_t *cm_base, const uint32_t *cm_scan,
                 Seg *W1, Seg *W8, SmallLists S, Seg *L2, Seg *E, uint2 *B, Seg *N,
                 Counters *c, int grid, cudaStream_t st) {
    const int g = grid_of(grid, nL, 1, 1u << 30);
    if (!g) return;
    k_emit<<<g, 256, 0, st>>>(a, L, nL, tile_base, nspl, cm_base, cm_scan, W1, W8, S, L2, E, B,
                              N, c);
}

// A span with host bounds and nothing in it launches nothing.
static bool span_empty(const Span &sp) {
    return !sp.lo.dev && !sp.hi.dev && sp.hi.host <= sp.lo.host;
}

void launch_warp1(const SortArgs &a, const Seg *W1, Span sp, Seg *N, Counters *c, int grid,
                  cudaStream_t st) {
    if (span_empty(sp) || grid <= 0) return;
    k_warp1<<<grid, WARP_THREADS, 0, st>>>(a, W1, sp, N, c);
}

void launch_warp8(const SortArgs &a, const Seg *W8, Span sp, Seg *N, Counters *c, int grid,
                  cudaStream_t st) {
    if (span_empty(sp) || grid <= 0) return;
    set_smem_attrs();
    k_warp8<<<grid, WARP_THREADS, W8_SMEM, st>>>(a, W8, sp, N, c);
}

void launch_block(const SortArgs &a, const Seg *S, Span sp, int cls, Seg *N, Counters *c,
                  int grid, cudaStream_t st, bool prefetch) {
    if (span_empty(sp) || grid <= 0) return;
    set_smem_attrs();
    if (prefetch) {
        if (cls == 0)
            k_block2<64><<<grid, SMALL_THREADS, BLOCK2_SMEM, st>>>(a, S, sp, N, c);
        else if (cls == 1)
            k_block2<128><<<grid, SMALL_THREADS, BLOCK2_SMEM, st>>>(a, S, sp, N, c);
        else
            k_block2<256><<<grid, SMALL_THREADS, BLOCK2_SMEM, st>>>(a, S, sp, N, c);
        return;
    }
#define SS_BLOCK_LAUNCH(VAR)                                                           \
    do {                                                                               \
        if (cls == 0)                                                                  \
            k_block<64, VAR><<<grid, SMALL_THREADS, BLOCK_SMEM, st>>>(a, S, sp, N, c);  \
        else if (cls == 1)                                                             \
            k_block<128, VAR><<<grid, SMALL_THREADS, BLOCK_SMEM, st>>>(a, S, sp, N, c); \
        else                                                                           \
            k_block<256, VAR><<<grid, SMALL_THREADS, BLOCK_SMEM, st>>>(a, S, sp, N, c); \
    } while (0)
    if (a.block_lean == 2)
        SS_BLOCK_LAUNCH(2);
    else if (a.block_lean == 1)
        SS_BLOCK_LAUNCH(1);
    else
        SS_BLOCK_LAUNCH(0);
#undef SS_BLOCK_LAUNCH
}

void launch_equal(const SortArgs &a, const Seg *E, Span sp, Seg *N, Counters *c, int grid,
                  cudaStream_t st) {
    if (span_empty(sp) || grid <= 0) return;
    k_equal<<<grid, 256, 0, st>>>(a, E, sp, N, c);
}

void launch_boundary(const SortArgs &a, const uint2 *B, Counters *c, int grid, cudaStream_t st) {
    k_boundary<<<grid, 256, 0, st>>>(a, B, c);
}

void launch_g_round_begin(GraphState *g, Counters *c, unsigned long long h_round,
                          cudaStream_t st) {
    k_g_round_begin<<<1, 128, 0, st>>>(g, c, (cudaGraphConditionalHandle)h_round);
}

void launch_g_after_classify(GraphState *g, Counters *c, unsigned long long h_level,
                             unsigned long long h_gather, cudaStream_t st) {
    k_g_after_classify<<<1, 32, 0, st>>>(g, c, (cudaGraphConditionalHandle)h_level,
                                         (cudaGraphConditionalHandle)h_gather);
}

void launch_g_level_begin(GraphState *g, unsigned long long h_level, unsigned long long h_first,
                          cudaStream_t st) {
    k_g_level_begin<<<1, 32, 0, st>>>(g, (cudaGraphConditionalHandle)h_level,
                                      (cudaGraphConditionalHandle)h_first);
}

void launch_g_level_end(GraphState *g, Counters *c, Seg *L, const Seg *L2,
                        unsigned long long h_level, int grid, cudaStream_t st) {
    k_g_level_end<<<grid, 256, 0, st>>>(g, c, L, L2, (cudaGraphConditionalHandle)h_level);
}

void launch_g_round_end(GraphState *g, Counters *c, Seg *R, const Seg *N,
                        unsigned long long h_round, int grid, cudaStream_t st) {
    k_g_round_end<<<grid, 256, 0, st>>>(g, c, R, N, (cudaGraphConditionalHandle)h_round);
}

}  // namespace ssort
