// ssort_kernels.cu -- sm_100a kernels of the MSD radix string sort.
//
// One refinement round works on the live segments at one depth (a multiple of
// 8 bytes).  For every live string it gathers the 8 bytes at arena[off+depth]
// as a big-endian key with every byte after the first NUL zeroed (the uint64
// form of the reference's get_char, src/util/get_char.h:68-89, but built with
// unsigned shifts; the reference's int-promoted shifts sign-extend bytes >= 0x80
// and are not reproduced).  Each segment is then sorted by (key, index):
// segments of <= 32 strings by one warp in registers, <= SMALL_CAP by one CTA
// in shared memory, larger ones are first split by sample partitioning into
// range buckets and equality buckets with a stable scatter.  Equal runs whose
// key holds no NUL (the reference's is_end test, src/util/get_char.h:162-175,
// and its bucket-skip rule, src/msd_ce.cpp:402) become the next round's
// segments at depth+8; every other adjacent pair gets its LCP here.
#include "ssort_internal.cuh"

namespace ssort {

namespace {

constexpr uint64_t KEY_MAX = ~0ull;
constexpr uint32_t IDX_MAX = ~0u;

__device__ __forceinline__ uint64_t bswap64(uint64_t x) {
    const uint32_t lo = (uint32_t)x, hi = (uint32_t)(x >> 32);
    return ((uint64_t)__byte_perm(lo, 0, 0x0123) << 32) | __byte_perm(hi, 0, 0x0123);
}

// 8 bytes of the string at arena[pos..], big-endian, zero after the first NUL.
__device__ __forceinline__ uint64_t load_key(const uint8_t *__restrict__ arena,
                                             uint64_t arena_bytes, uint64_t pos) {
    uint64_t w;
    const uint64_t a = pos & ~7ull;
    const uint32_t sh = (uint32_t)(pos & 7) * 8;
    if (a + 16 <= arena_bytes) {
        const uint64_t *p = reinterpret_cast<const uint64_t *>(arena + a);
        const uint64_t lo = __ldg(p);
        if (sh) {
            const uint64_t hi = __ldg(p + 1);
            w = (lo >> sh) | (hi << (64 - sh));
        } else {
            w = lo;
        }
    } else {
        // Within 16 bytes of the arena end: byte loads, never past the end
        // (bytes past the end read as NUL).
        w = 0;
        for (int i = 0; i < 8; ++i) {
            const uint64_t q = pos + i;
            if (q >= arena_bytes) break;
            const uint8_t c = arena[q];
            w |= (uint64_t)c << (8 * i);
            if (!c) break;
        }
    }
    // Little-endian word: byte 0 is arena[pos].  The lowest flagged byte of
    // the classic zero-byte test is the first NUL (no false positives below it).
    const uint64_t z = (w - 0x0101010101010101ull) & ~w & 0x8080808080808080ull;
    if (z) {
        const uint32_t jb = (uint32_t)(__ffsll((long long)z) - 1) >> 3;
        w &= jb ? ((1ull << (8 * jb)) - 1) : 0ull;
    }
    return bswap64(w);
}

// The key holds the end of its string (low byte NUL).
__device__ __forceinline__ bool key_is_end(uint64_t k) { return (k & 0xFF) == 0; }

// Number of string bytes in a key that contains the NUL.
__device__ __forceinline__ uint32_t key_len(uint64_t k) {
    return k ? 8u - ((uint32_t)(__ffsll((long long)k) - 1) >> 3) : 0u;
}

// LCP contribution of two keys at the same depth (reference lcp(),
// src/mergesort_lcp.cpp:88-100: stop at the first difference or the NUL).
__device__ __forceinline__ uint32_t key_lcp(uint64_t a, uint64_t b) {
    return a == b ? key_len(a) : ((uint32_t)__clzll((long long)(a ^ b)) >> 3);
}

__device__ __forceinline__ uint64_t string_offset(const void *offs, int off_width, uint32_t i) {
    return off_width == 8 ? __ldg(reinterpret_cast<const unsigned long long *>(offs) + i)
                          : (uint64_t)__ldg(reinterpret_cast<const uint32_t *>(offs) + i);
}

__device__ __forceinline__ bool pair_less(uint64_t ka, uint32_t ia, uint64_t kb, uint32_t ib) {
    return ka < kb || (ka == kb && ia < ib);
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

__device__ __forceinline__ void emit_next(Seg *N, Counters *c, uint32_t start, uint32_t len,
                                          uint32_t depth) {
    const uint32_t slot = atomicAdd(&c->n_next, 1u);
    N[slot] = Seg{start, len, depth, 0u};
    atomicAdd(&c->live_next, (unsigned long long)len);
}

// Bucket of `key` among u sorted distinct splitters s[0..u) padded with
// KEY_MAX to kp2-1 entries: range bucket 2j holds s[j-1] < key < s[j],
// equality bucket 2j+1 holds key == s[j].
__device__ __forceinline__ uint32_t classify(const uint64_t *s, uint32_t kp2, uint32_t u,
                                             uint64_t key) {
    uint32_t lo = 0;
    for (uint32_t step = kp2 >> 1; step > 0; step >>= 1)
        if (s[lo + step - 1] < key) lo += step;
    return (lo < u && s[lo] == key) ? 2 * lo + 1 : 2 * lo;
}

// ---------------------------------------------------------------------------
__global__ void k_iota(uint32_t *idx, uint32_t n) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        idx[i] = i;
}

__global__ void k_classify(const Seg *__restrict__ R, uint32_t nR, Seg *T, Seg *S, Seg *L,
                           Counters *c) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nR) return;
    const Seg s = R[i];
    if (s.len <= (uint32_t)TINY_CAP)
        T[atomicAdd(&c->n_tiny, 1u)] = s;
    else if (s.len <= (uint32_t)SMALL_CAP)
        S[atomicAdd(&c->n_small, 1u)] = s;
    else {
        L[atomicAdd(&c->n_large, 1u)] = s;
        atomicAdd(&c->gather_elems, (unsigned long long)s.len);
    }
}

__global__ void k_tile_counts(const Seg *__restrict__ segs, uint32_t n, uint32_t tile,
                              uint32_t *out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = (segs[i].len + tile - 1) / tile;
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
                                                              uint32_t n, uint32_t *partials) {
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_CHUNK;
    uint32_t s = 0;
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        const uint64_t i = base + (uint64_t)k * SCAN_THREADS + threadIdx.x;
        if (i < n) s += in[i];
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
                                                            uint32_t n,
                                                            const uint32_t *__restrict__ partials,
                                                            uint32_t nparts) {
    __shared__ uint32_t buf[SCAN_CHUNK];
    const uint64_t base = (uint64_t)blockIdx.x * SCAN_CHUNK;
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
    if (blockIdx.x == 0 && threadIdx.x == 0) out[n] = partials[nparts];
}

// ---- key gather for large segments ----------------------------------------
__global__ void __launch_bounds__(GATHER_THREADS) k_gather(SortArgs a, const Seg *__restrict__ L,
                                                          uint32_t nL,
                                                          const uint32_t *__restrict__ tile_base,
                                                          uint32_t total_tiles) {
    constexpr int U = GATHER_TILE / GATHER_THREADS;
    for (uint32_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint32_t si = find_seg(tile_base, nL, t);
        const Seg s = L[si];
        const uint32_t lo = (t - tile_base[si]) * GATHER_TILE;
        const uint32_t *I = a.idx[0];
        uint32_t id[U];
        uint64_t off[U];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = lo + u * GATHER_THREADS + threadIdx.x;
            id[u] = i < s.len ? I[s.start + i] : IDX_MAX;
        }
#pragma unroll
        for (int u = 0; u < U; ++u)
            off[u] = id[u] != IDX_MAX ? string_offset(a.offs, a.off_width, id[u]) : 0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const uint32_t i = lo + u * GATHER_THREADS + threadIdx.x;
            if (id[u] != IDX_MAX)
                a.key[0][s.start + i] = load_key(a.arena, a.arena_bytes, off[u] + s.depth);
        }
    }
}

// ---- splitter selection: one CTA per large segment ------------------------
constexpr int SAMPLE_THREADS = 512;

__device__ __forceinline__ uint32_t hash32(uint32_t x) {
    x ^= x >> 16;
    x *= 0x7feb352du;
    x ^= x >> 15;
    x *= 0x846ca68bu;
    x ^= x >> 16;
    return x;
}

__global__ void __launch_bounds__(SAMPLE_THREADS) k_sample(SortArgs a, const Seg *__restrict__ L,
                                                           uint64_t *spl, uint32_t *nspl,
                                                           uint32_t *ntiles, uint32_t *cm_size) {
    __shared__ uint64_t smp[SAMPLES];
    __shared__ uint32_t keep[SAMPLE_THREADS + 1];
    const Seg s = L[blockIdx.x];
    const uint64_t *K = a.keyb(s.flags & SEG_BUF1);
    for (int i = threadIdx.x; i < SAMPLES; i += SAMPLE_THREADS) {
        const uint32_t r = hash32(s.start * 0x9E3779B1u + (uint32_t)i * 0x85EBCA77u + s.len);
        const uint32_t p = (uint32_t)(((uint64_t)r * s.len) >> 32);
        smp[i] = K[s.start + p];
    }
    __syncthreads();
    for (int k = 2; k <= SAMPLES; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < SAMPLES; i += SAMPLE_THREADS) {
                const int l = i ^ j;
                if (l > i) {
                    const uint64_t x = smp[i], y = smp[l];
                    const bool asc = (i & k) == 0;
                    if ((x > y) == asc) {
                        smp[i] = y;
                        smp[l] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    // k candidate splitters at evenly spaced sample ranks, deduplicated.
    uint32_t k = (s.len + SMALL_CAP / 4 - 1) / (SMALL_CAP / 4);
    if (k > (uint32_t)KMAX) k = KMAX;
    if (k < 1) k = 1;
    uint64_t *out = spl + (uint64_t)blockIdx.x * SPL_STRIDE;
    // Thread j < k owns candidate j; it survives if it differs from j-1.
    // Compact survivors with a block scan over SAMPLE_THREADS >= KMAX slots.
    const uint32_t j = threadIdx.x;
    uint64_t cand = 0;
    uint32_t flag = 0;
    if (j < k) {
        cand = smp[((uint64_t)(j + 1) * SAMPLES) / (k + 1)];
        flag = (j == 0) || smp[((uint64_t)j * SAMPLES) / (k + 1)] != cand;
    }
    keep[j] = flag;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t run = 0;
        for (uint32_t q = 0; q < (uint32_t)SAMPLE_THREADS; ++q) {
            const uint32_t f = keep[q];
            keep[q] = run;
            run += f;
        }
        keep[SAMPLE_THREADS] = run;
    }
    __syncthreads();
    const uint32_t u = keep[SAMPLE_THREADS];
    if (flag) out[keep[j]] = cand;
    const uint32_t kp2 = next_pow2(u + 1);
    for (uint32_t q = u + threadIdx.x; q < kp2 - 1; q += SAMPLE_THREADS) out[q] = KEY_MAX;
    if (threadIdx.x == 0) {
        nspl[blockIdx.x] = u;
        const uint32_t nt = (s.len + PART_TILE - 1) / PART_TILE;
        ntiles[blockIdx.x] = nt;
        cm_size[blockIdx.x] = (2 * u + 1) * nt;
    }
}

// ---- partition count: per-tile bucket histograms ---------------------------
__global__ void __launch_bounds__(PART_THREADS) k_count(SortArgs a, const Seg *__restrict__ L,
                                                        uint32_t nL,
                                                        const uint32_t *__restrict__ tile_base,
                                                        uint32_t total_tiles,
                                                        const uint64_t *__restrict__ spl,
                                                        const uint32_t *__restrict__ nspl,
                                                        const uint32_t *__restrict__ cm_base,
                                                        uint32_t *cm) {
    __shared__ uint64_t sspl[SPL_STRIDE];
    __shared__ uint32_t hist[NB_MAX + 1];
    for (uint32_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint32_t si = find_seg(tile_base, nL, t);
        const Seg s = L[si];
        const uint32_t u = nspl[si], kp2 = next_pow2(u + 1), nb = 2 * u + 1;
        for (uint32_t q = threadIdx.x; q + 1 < kp2; q += PART_THREADS)
            sspl[q] = spl[(uint64_t)si * SPL_STRIDE + q];
        for (uint32_t q = threadIdx.x; q < nb; q += PART_THREADS) hist[q] = 0;
        __syncthreads();
        const uint32_t tl = t - tile_base[si];
        const uint32_t nt = tile_base[si + 1] - tile_base[si];
        const uint32_t lo = tl * PART_TILE;
        const uint64_t *K = a.keyb(s.flags & SEG_BUF1) + s.start;
#pragma unroll 4
        for (int it = 0; it < PART_ITEMS; ++it) {
            const uint32_t i = lo + it * PART_THREADS + threadIdx.x;
            if (i < s.len) atomicAdd(&hist[classify(sspl, kp2, u, K[i])], 1u);
        }
        __syncthreads();
        for (uint32_t q = threadIdx.x; q < nb; q += PART_THREADS)
            cm[cm_base[si] + (uint64_t)q * nt + tl] = hist[q];
        __syncthreads();
    }
}

// ---- partition scatter: stable within and across tiles ---------------------
__global__ void __launch_bounds__(PART_THREADS) k_scatter(SortArgs a, const Seg *__restrict__ L,
                                                          uint32_t nL,
                                                          const uint32_t *__restrict__ tile_base,
                                                          uint32_t total_tiles,
                                                          const uint64_t *__restrict__ spl,
                                                          const uint32_t *__restrict__ nspl,
                                                          const uint32_t *__restrict__ cm_base,
                                                          const uint32_t *__restrict__ cm_scan) {
    __shared__ uint64_t sspl[SPL_STRIDE];
    __shared__ uint32_t wcnt[PART_WARPS][NB_MAX + 1];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    constexpr int SUB = PART_TILE / PART_WARPS;  // consecutive keys per warp
    for (uint32_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint32_t si = find_seg(tile_base, nL, t);
        const Seg s = L[si];
        const uint32_t u = nspl[si], kp2 = next_pow2(u + 1), nb = 2 * u + 1;
        const uint32_t tl = t - tile_base[si];
        const uint32_t nt = tile_base[si + 1] - tile_base[si];
        const uint32_t lo = tl * PART_TILE;
        for (uint32_t q = threadIdx.x; q + 1 < kp2; q += PART_THREADS)
            sspl[q] = spl[(uint64_t)si * SPL_STRIDE + q];
        for (uint32_t q = threadIdx.x; q <= nb; q += PART_THREADS)
#pragma unroll
            for (int ww = 0; ww < PART_WARPS; ++ww) wcnt[ww][q] = 0;
        const int ib = s.flags & SEG_BUF1;
        const uint64_t *Kin = a.keyb(ib) + s.start;
        const uint32_t *Iin = a.idxb(ib) + s.start;
        uint64_t *Kout = a.keyb(ib ^ 1) + s.start;
        uint32_t *Iout = a.idxb(ib ^ 1) + s.start;
        uint64_t kk[PART_ITEMS];
        uint32_t ii[PART_ITEMS];
        uint32_t br[PART_ITEMS];
#pragma unroll
        for (int c = 0; c < PART_ITEMS; ++c) {
            const uint32_t e = lo + w * SUB + c * 32 + lane;
            const bool v = e < s.len;
            kk[c] = v ? Kin[e] : 0;
            ii[c] = v ? Iin[e] : 0;
        }
        __syncthreads();
        const uint32_t lt = lanemask_lt();
#pragma unroll
        for (int c = 0; c < PART_ITEMS; ++c) {
            const uint32_t e = lo + w * SUB + c * 32 + lane;
            const uint32_t b = e < s.len ? classify(sspl, kp2, u, kk[c]) : nb;
            const uint32_t peers = __match_any_sync(0xffffffffu, b);
            const uint32_t r = __popc(peers & lt);
            const uint32_t base = wcnt[w][b];
            __syncwarp();
            if (r == 0) wcnt[w][b] = base + __popc(peers);
            __syncwarp();
            br[c] = (b << 16) | (base + r);
        }
        __syncthreads();
        // Exclusive scan over warps per bucket, plus the tile's global base.
        const uint32_t cmb = cm_base[si];
        const uint32_t seg0 = cm_scan[cmb];
        for (uint32_t q = threadIdx.x; q < nb; q += PART_THREADS) {
            uint32_t run = cm_scan[cmb + (uint64_t)q * nt + tl] - seg0;
#pragma unroll
            for (int ww = 0; ww < PART_WARPS; ++ww) {
                const uint32_t x = wcnt[ww][q];
                wcnt[ww][q] = run;
                run += x;
            }
        }
        __syncthreads();
#pragma unroll
        for (int c = 0; c < PART_ITEMS; ++c) {
            const uint32_t e = lo + w * SUB + c * 32 + lane;
            if (e < s.len) {
                const uint32_t b = br[c] >> 16;
                const uint32_t o = wcnt[w][b] + (br[c] & 0xFFFF);
                Kout[o] = kk[c];
                Iout[o] = ii[c];
            }
        }
        __syncthreads();
    }
}

// ---- bucket emission: one CTA per partitioned segment ----------------------
__global__ void k_emit(SortArgs a, const Seg *__restrict__ L, const uint32_t *__restrict__ tile_base,
                       const uint32_t *__restrict__ nspl, const uint32_t *__restrict__ cm_base,
                       const uint32_t *__restrict__ cm_scan, Seg *T, Seg *S, Seg *L2, Seg *E,
                       uint2 *B, Counters *c) {
    const uint32_t si = blockIdx.x;
    const Seg s = L[si];
    const uint32_t u = nspl[si], nb = 2 * u + 1;
    const uint32_t nt = tile_base[si + 1] - tile_base[si];
    const uint32_t cmb = cm_base[si];
    const uint32_t seg0 = cm_scan[cmb];
    const uint32_t ob = (s.flags & SEG_BUF1) ^ 1u;
    const uint32_t flags = ob | SEG_KEYS;
    for (uint32_t b = threadIdx.x; b < nb; b += blockDim.x) {
        const uint32_t off = cm_scan[cmb + (uint64_t)b * nt] - seg0;
        const uint32_t end = b + 1 < nb ? cm_scan[cmb + (uint64_t)(b + 1) * nt] - seg0 : s.len;
        const uint32_t len = end - off;
        if (len == 0) continue;
        const uint32_t p = s.start + off;
        if (off > 0) B[atomicAdd(&c->n_bound, 1u)] = make_uint2(p, s.depth);
        if (len == 1) {
            if (ob) {
                a.idx[0][p] = a.idx[1][p];
                a.key[0][p] = a.key[1][p];
            }
            continue;
        }
        const Seg o{p, len, s.depth, flags};
        if (b & 1) {
            E[atomicAdd(&c->n_equal, 1u)] = Seg{p, len, s.depth, flags | SEG_EQUAL};
        } else if (len <= (uint32_t)TINY_CAP) {
            T[atomicAdd(&c->n_tiny, 1u)] = o;
        } else if (len <= (uint32_t)SMALL_CAP) {
            S[atomicAdd(&c->n_small, 1u)] = o;
        } else {
            L2[atomicAdd(&c->n_large_next, 1u)] = o;
        }
    }
    if (threadIdx.x == 0) atomicAdd(&c->partitioned, (unsigned long long)s.len);
}

// ---- tiny segments: one warp, bitonic sort in registers --------------------
constexpr int TINY_THREADS = 256;

__global__ void __launch_bounds__(TINY_THREADS) k_tiny(SortArgs a, const Seg *__restrict__ T,
                                                       uint32_t nT, Seg *N, Counters *c) {
    const int lane = threadIdx.x & 31;
    const uint32_t warp0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    unsigned long long fresh = 0, keyed = 0;
    for (uint32_t g = warp0; g < nT; g += nwarps) {
        const Seg s = T[g];
        const int b = s.flags & SEG_BUF1;
        const bool v = (uint32_t)lane < s.len;
        if (s.flags & SEG_KEYS)
            keyed += s.len;
        else
            fresh += s.len;
        uint32_t id = IDX_MAX;
        uint64_t k = KEY_MAX;
        if (v) {
            id = a.idxb(b)[s.start + lane];
            k = (s.flags & SEG_KEYS)
                    ? a.keyb(b)[s.start + lane]
                    : load_key(a.arena, a.arena_bytes,
                               string_offset(a.offs, a.off_width, id) + s.depth);
        }
#pragma unroll
        for (int kk = 2; kk <= 32; kk <<= 1) {
#pragma unroll
            for (int j = kk >> 1; j > 0; j >>= 1) {
                const uint64_t ok = __shfl_xor_sync(0xffffffffu, k, j);
                const uint32_t oi = __shfl_xor_sync(0xffffffffu, id, j);
                const bool want_min = ((lane & j) == 0) == ((lane & kk) == 0);
                const bool other_less = pair_less(ok, oi, k, id);
                const bool other_more = pair_less(k, id, ok, oi);
                if (want_min ? other_less : other_more) {
                    k = ok;
                    id = oi;
                }
            }
        }
        const uint64_t prev = __shfl_up_sync(0xffffffffu, k, 1);
        const uint64_t next = __shfl_down_sync(0xffffffffu, k, 1);
        const bool head = v && (lane == 0 || prev != k);
        const uint32_t heads = __ballot_sync(0xffffffffu, head);
        if (v) {
            const uint32_t p = s.start + lane;
            a.idx[0][p] = id;
            if (lane == 0 || (uint32_t)lane == s.len - 1) a.key[0][p] = k;
            if (lane > 0) {
                if (prev != k)
                    a.lcp[p] = s.depth + key_lcp(prev, k);
                else if (key_is_end(k))
                    a.lcp[p] = s.depth + key_len(k);
            }
            const bool tail = (uint32_t)lane == s.len - 1 || next != k;
            if (tail && !head && !key_is_end(k)) {
                const uint32_t m = lane == 31 ? 0xffffffffu : ((2u << lane) - 1u);
                const uint32_t h = 31 - __clz(heads & m);
                emit_next(N, c, s.start + h, lane - h + 1, s.depth + 8);
            }
        }
    }
    if (lane == 0 && (fresh | keyed)) {
        atomicAdd(&c->tiny_fresh, fresh);
        atomicAdd(&c->tiny_keyed, keyed);
    }
}

// ---- small segments: one CTA, bitonic sort in shared memory -----------------
__global__ void __launch_bounds__(SMALL_THREADS) k_small(SortArgs a, const Seg *__restrict__ S,
                                                         uint32_t nS, Seg *N, Counters *c) {
    __shared__ uint64_t sk[SMALL_CAP];
    __shared__ uint32_t sx[SMALL_CAP];
    unsigned long long fresh = 0, keyed = 0;
    for (uint32_t g = blockIdx.x; g < nS; g += gridDim.x) {
        const Seg s = S[g];
        const int b = s.flags & SEG_BUF1;
        const uint32_t P = next_pow2(s.len);
        if (s.flags & SEG_KEYS)
            keyed += s.len;
        else
            fresh += s.len;
        for (uint32_t i = threadIdx.x; i < P; i += SMALL_THREADS) {
            if (i < s.len) {
                const uint32_t id = a.idxb(b)[s.start + i];
                sx[i] = id;
                sk[i] = (s.flags & SEG_KEYS)
                            ? a.keyb(b)[s.start + i]
                            : load_key(a.arena, a.arena_bytes,
                                       string_offset(a.offs, a.off_width, id) + s.depth);
            } else {
                sx[i] = IDX_MAX;
                sk[i] = KEY_MAX;
            }
        }
        __syncthreads();
        for (uint32_t k = 2; k <= P; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < P; i += SMALL_THREADS) {
                    const uint32_t l = i ^ j;
                    if (l > i) {
                        const uint64_t ki = sk[i], kl = sk[l];
                        const uint32_t xi = sx[i], xl = sx[l];
                        const bool asc = (i & k) == 0;
                        if (pair_less(kl, xl, ki, xi) == asc) {
                            sk[i] = kl;
                            sk[l] = ki;
                            sx[i] = xl;
                            sx[l] = xi;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t i = threadIdx.x; i < s.len; i += SMALL_THREADS) {
            const uint32_t p = s.start + i;
            const uint64_t k = sk[i];
            a.idx[0][p] = sx[i];
            if (i == 0 || i == s.len - 1) a.key[0][p] = k;
            const bool same_prev = i > 0 && sk[i - 1] == k;
            if (i > 0) {
                if (!same_prev)
                    a.lcp[p] = s.depth + key_lcp(sk[i - 1], k);
                else if (key_is_end(k))
                    a.lcp[p] = s.depth + key_len(k);
            }
            const bool tail = i == s.len - 1 || sk[i + 1] != k;
            if (tail && same_prev && !key_is_end(k)) {
                // First position of this run: lower bound of k in sk[0..i].
                uint32_t lo = 0, hi = i;
                while (lo < hi) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (sk[mid] < k)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                emit_next(N, c, s.start + lo, i - lo + 1, s.depth + 8);
            }
        }
        __syncthreads();
    }
    if (threadIdx.x == 0 && (fresh | keyed)) {
        atomicAdd(&c->small_fresh, fresh);
        atomicAdd(&c->small_keyed, keyed);
    }
}

// ---- equality buckets ------------------------------------------------------
__global__ void k_equal(SortArgs a, const Seg *__restrict__ E, uint32_t nE,
                        const uint32_t *__restrict__ tile_base, uint32_t total_tiles, Seg *N,
                        Counters *c) {
    unsigned long long moved = 0, fin = 0;
    for (uint32_t t = blockIdx.x; t < total_tiles; t += gridDim.x) {
        const uint32_t si = find_seg(tile_base, nE, t);
        const Seg s = E[si];
        const int b = s.flags & SEG_BUF1;
        const uint64_t k = a.keyb(b)[s.start];
        const bool end = key_is_end(k);
        const uint32_t tl = t - tile_base[si];
        if (tl == 0 && threadIdx.x == 0) {
            a.key[0][s.start] = k;
            a.key[0][s.start + s.len - 1] = k;
            if (!end) emit_next(N, c, s.start, s.len, s.depth + 8);
        }
        if (!b && !end) continue;
        const uint32_t lo = tl * EQ_TILE;
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

__global__ void k_boundary(SortArgs a, const uint2 *__restrict__ B, uint32_t nB) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nB) return;
    const uint2 e = B[i];
    a.lcp[e.x] = e.y + key_lcp(a.key[0][e.x - 1], a.key[0][e.x]);
}

}  // namespace

// ---- launchers --------------------------------------------------------------
static inline uint32_t cdiv(uint64_t a, uint64_t b) { return (uint32_t)((a + b - 1) / b); }

void launch_iota(uint32_t *idx, uint32_t n, cudaStream_t st) {
    const uint32_t g = cdiv(n, 256) < 148 * 16 ? cdiv(n, 256) : 148 * 16;
    k_iota<<<g ? g : 1, 256, 0, st>>>(idx, n);
}

void launch_classify(const Seg *R, uint32_t nR, Seg *T, Seg *S, Seg *L, Counters *c,
                     cudaStream_t st) {
    if (!nR) return;
    k_classify<<<cdiv(nR, 256), 256, 0, st>>>(R, nR, T, S, L, c);
}

void launch_tile_counts(const Seg *segs, uint32_t n, uint32_t tile, uint32_t *out,
                        cudaStream_t st) {
    if (!n) return;
    k_tile_counts<<<cdiv(n, 256), 256, 0, st>>>(segs, n, tile, out);
}

uint32_t scan_partials_needed(uint32_t n) { return cdiv(n ? n : 1, SCAN_CHUNK) + 1; }

void launch_scan(const uint32_t *in, uint32_t *out, uint32_t n, uint32_t *partials,
                 cudaStream_t st) {
    const uint32_t nb = cdiv(n ? n : 1, SCAN_CHUNK);
    k_scan_reduce<<<nb, SCAN_THREADS, 0, st>>>(in, n, partials);
    k_scan_partials<<<1, SCAN_THREADS, 0, st>>>(partials, nb);
    k_scan_down<<<nb, SCAN_THREADS, 0, st>>>(in, out, n, partials, nb);
}

void launch_gather(const SortArgs &a, const Seg *L, uint32_t nL, const uint32_t *tile_base,
                   uint32_t total_tiles, int grid, cudaStream_t st) {
    if (!total_tiles) return;
    k_gather<<<grid, GATHER_THREADS, 0, st>>>(a, L, nL, tile_base, total_tiles);
}

void launch_sample(const SortArgs &a, const Seg *L, uint32_t nL, uint64_t *spl, uint32_t *nspl,
                   uint32_t *ntiles, uint32_t *cm_size, cudaStream_t st) {
    if (!nL) return;
    k_sample<<<nL, SAMPLE_THREADS, 0, st>>>(a, L, spl, nspl, ntiles, cm_size);
}

void launch_count(const SortArgs &a, const Seg *L, uint32_t nL, const uint32_t *tile_base,
                  uint32_t total_tiles, const uint64_t *spl, const uint32_t *nspl,
                  const uint32_t *cm_base, uint32_t *cm, int grid, cudaStream_t st) {
    if (!total_tiles) return;
    k_count<<<grid, PART_THREADS, 0, st>>>(a, L, nL, tile_base, total_tiles, spl, nspl, cm_base,
                                           cm);
}

void launch_scatter(const SortArgs &a, const Seg *L, uint32_t nL, const uint32_t *tile_base,
                    uint32_t total_tiles, const uint64_t *spl, const uint32_t *nspl,
                    const uint32_t *cm_base, const uint32_t *cm_scan, int grid,
                    cudaStream_t st) {
    if (!total_tiles) return;
    k_scatter<<<grid, PART_THREADS, 0, st>>>(a, L, nL, tile_base, total_tiles, spl, nspl,
                                             cm_base, cm_scan);
}

void launch_emit(const SortArgs &a, const Seg *L, uint32_t nL, const uint32_t *tile_base,
                 const uint32_t *nspl, const uint32_t *cm_base, const uint32_t *cm_scan,
                 Seg *T, Seg *S, Seg *L2, Seg *E, uint2 *B, Counters *c, cudaStream_t st) {
    if (!nL) return;
    k_emit<<<nL, 256, 0, st>>>(a, L, tile_base, nspl, cm_base, cm_scan, T, S, L2, E, B, c);
}

void launch_tiny(const SortArgs &a, const Seg *T, uint32_t nT, Seg *N, Counters *c, int grid,
                 cudaStream_t st) {
    if (!nT) return;
    const uint32_t need = cdiv(nT, TINY_THREADS / 32);
    k_tiny<<<need < (uint32_t)grid ? need : (uint32_t)grid, TINY_THREADS, 0, st>>>(a, T, nT, N, c);
}

void launch_small(const SortArgs &a, const Seg *S, uint32_t nS, Seg *N, Counters *c, int grid,
                  cudaStream_t st) {
    if (!nS) return;
    k_small<<<nS < (uint32_t)grid ? nS : (uint32_t)grid, SMALL_THREADS, 0, st>>>(a, S, nS, N, c);
}

void launch_equal(const SortArgs &a, const Seg *E, uint32_t nE, const uint32_t *tile_base,
                  uint32_t total_tiles, Seg *N, Counters *c, int grid, cudaStream_t st) {
    if (!total_tiles) return;
    const uint32_t g = total_tiles < (uint32_t)grid ? total_tiles : (uint32_t)grid;
    k_equal<<<g, 256, 0, st>>>(a, E, nE, tile_base, total_tiles, N, c);
}

void launch_boundary(const SortArgs &a, const uint2 *B, uint32_t nB, cudaStream_t st) {
    if (!nB) return;
    k_boundary<<<cdiv(nB, 256), 256, 0, st>>>(a, B, nB);
}

}  // namespace ssort
