// ssort_internal.cuh -- types, tuning constants and kernel launchers shared by
// the device code (ssort_kernels.cu) and the host engine (ssort_engine.cu).
//
// Data layout in HBM for one sort of n strings:
//   arena            the string bytes (read-only), NUL-terminated strings,
//                    16-byte aligned base
//   offs[n]          uint32 or uint64 offset of string i in the arena
//   idx[0], idx[1]   uint32 string indices in sorted-position order (ping-pong);
//                    idx[0] is the caller's perm buffer and holds the result
//   key[0], key[1]   16-byte big-endian key (two uint64 words, most
//                    significant first) of each live position at the depth of
//                    its segment, every byte after the first NUL zeroed
//                    (ping-pong with idx)
//   lcp[n]           uint32 LCP array (the caller's buffer or an internal one)
//   segment lists    Seg records; every live segment is a contiguous range of
//                    positions whose strings agree on their first `depth` bytes
//                    and sit in ascending index order (so sorting by
//                    (key, index) is exactly a stable sort by key).
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ssort {

// Bytes of string consumed per refinement round.
constexpr uint32_t KEY_BYTES = 16;

// Seg.flags
constexpr uint32_t SEG_BUF1 = 1u;   // idx/keys of this segment live in buffer 1
constexpr uint32_t SEG_KEYS = 2u;   // key[buf] already holds this depth's keys
constexpr uint32_t SEG_CHUNK_SHIFT = 8;  // equality work items: chunk index << 8

struct Seg {
    uint32_t start, len, depth, flags;
};

// Segments of at most WARP1_CAP strings are sorted by one warp with one string
// per lane, at most WARP8_CAP (or the runtime cutoff below it) by one warp
// with up to 8 strings per lane, at most SMALL_CAP by a thread group of a CTA;
// larger ones are split by sample partitioning first.
constexpr int WARP1_CAP = 32;
constexpr int WARP8_CAP = 256;
constexpr uint32_t WARP1_DEEP = 64;       // default in-warp refinement steps (16 bytes each)
constexpr uint32_t WARP1_DEEP_MAX = 4096;
constexpr uint32_t KEY2_MIN_N = 1u << 20;           // sorts that may save round-1 keys
constexpr uint64_t NARROW_OFFS_MIN_N = 1u << 20;    // host sorts that narrow 8-byte offsets
constexpr uint32_t KEY2_MIN_BYTES_PER_STRING = 24;  // ... when the arena has this many
constexpr double KEY2_MIN_ROUND1_LIVE = 0.25;       // ... and the last sort's round-1 share
constexpr int SMALL_CAP = 2048;
constexpr int SMALL_THREADS = 256;
constexpr int SMALL_ITEMS = SMALL_CAP / SMALL_THREADS;  // 8
// The CTA sort splits its segments into three size classes, sorted by groups
// of 64, 128 and 256 threads (8 strings per thread): <= BLOCK_CAP1,
// <= BLOCK_CAP2 and <= SMALL_CAP strings.
constexpr int BLOCK_CAP1 = 512;
constexpr int BLOCK_CAP2 = 1024;

// Sample partitioning of large segments.
constexpr int KMAX = 511;               // splitters per segment and pass
constexpr int SPL_STRIDE = 512;         // splitter slots per segment (pow2)
// Splitter lookup table: for the 12 key bits after the splitters' common
// prefix, the index range of splitters carrying those bits.
constexpr int TBL_BITS = 12;
constexpr int TBL_N = 1 << TBL_BITS;
constexpr int TBL_STRIDE = TBL_N + 64;  // uint16 entries per segment (TBL_N + 1 used)
constexpr int NB_MAX = 2 * KMAX + 1;    // range + equality buckets
constexpr int SAMPLES_MAX = 4096;       // keys sampled per large segment
constexpr int TARGET_BUCKET = 512;      // default wanted strings per range bucket
constexpr int PART_THREADS = 512;
constexpr int PART_WARPS = PART_THREADS / 32;
constexpr int PART_ITEMS = 8;
constexpr int PART_TILE = PART_THREADS * PART_ITEMS;  // 4096 keys per tile

constexpr int GATHER_TILE = 4096;
constexpr int GATHER_THREADS = 256;
constexpr int GATHER_ITEMS = 8;
constexpr int EQ_TILE = 8192;

struct Counters {
    uint32_t n_w1, n_w8, n_small, n_large;
    uint32_t n_equal, n_bound, n_next, n_large_next;
    uint32_t gather_tiles, part_tiles, cm_total, error;
    unsigned long long live_next;    // strings in next-round segments
    unsigned long long partitioned;  // strings moved by partition scatters
    // element counts per kernel (for the algorithmic-bytes roofline)
    unsigned long long gather_elems;  // keys gathered by k_gather
    unsigned long long warp1_fresh, warp1_keyed, warp8_fresh, warp8_keyed, block_fresh,
        block_keyed;
    unsigned long long equal_moved, equal_final;  // equality-bucket copies / lcp fills
    uint32_t n_small2, n_small3;  // CTA-sort segments of the 2nd and 3rd size class
    unsigned long long warp1_deep;  // strings re-sorted by in-warp refinement steps
    unsigned long long full_sorted;  // strings of segments re-sorted by the full comparator
    unsigned long long window_saved, window_used;  // key2 entries written / read
};

// A count the host knows (dev == nullptr: `host`) or only the device knows:
// *dev, or dev[*at] when `at` is set (a count stored at an index that is
// itself a device value).  The host-driven round loop passes host counts;
// the device-driven loop (a CUDA graph whose kernels find their work in
// device memory) passes device ones.
struct Count {
    uint32_t host;
    const uint32_t *dev;
    const uint32_t *at;
};
inline Count hcount(uint32_t n) { return Count{n, nullptr, nullptr}; }
inline Count dcount(const uint32_t *d, const uint32_t *at = nullptr) { return Count{0, d, at}; }
#ifdef __CUDACC__
__device__ __forceinline__ uint32_t count_of(const Count &c) {
    return c.dev ? (c.at ? c.dev[*c.at] : *c.dev) : c.host;
}
#endif
// Entries [lo, hi) of a segment list.
struct Span {
    Count lo, hi;
};
inline Span hspan(uint32_t lo, uint32_t hi) { return Span{hcount(lo), hcount(hi)}; }

// The CTA-sort segment lists, one per size class (n_small, n_small2, n_small3).
struct SmallLists {
    Seg *s[3];
};

struct SortArgs {
    __device__ __forceinline__ uint32_t *idxb(int b) const { return b ? idx[1] : idx[0]; }
    __device__ __forceinline__ ulonglong2 *keyb(int b) const { return b ? key[1] : key[0]; }

    const uint8_t *arena;
    uint64_t arena_bytes;
    const void *offs;
    int off_width;
    uint32_t n;
    uint32_t *idx[2];
    ulonglong2 *key[2];
    uint32_t *lcp;
    uint32_t *bkt;  // per position during a partition level: bucket << 12 | offset
    uint32_t target_bucket;  // wanted strings per range bucket of a partition
    uint32_t warp8_cap;      // largest segment for the one-warp sort (64..WARP8_CAP)
    uint32_t warp1_deep;     // in-warp refinement steps of the one-per-lane sort
    uint32_t l2_prefetch;    // partition kernels stream their next tile into L2 ahead
    uint32_t scatter_staged_idx;  // 0: k_scatter; 1: indices only (k_scatter2); 2: bulk key runs
    uint32_t block_lean;     // CTA sort: neighbour LCPs from the packed windows
    uint32_t match_vote;     // count kernel ranks with ballots instead of the match unit
    uint32_t warp_merge;     // warp sorts of packed keys: local networks + merge passes
    uint32_t max_splitters;  // splitters per partition pass, 2^(digit bits - 1) - 1 <= KMAX
    // Per segment size class (floor(log2 len)): the wanted strings per range
    // bucket autotuned for that class (0: target_bucket).  Set for batched
    // sorts, whose instances and segments span many size classes.
    uint16_t target_by_class[32];
    // Per string id, key bytes 16..31 as round 0's gather read them (it reads
    // those sectors of the arena anyway); round 1's first partition level
    // takes its keys from here instead of the offset and a random arena read.
    // Null when not in use.
    ulonglong2 *key2;
};

// ---- device-driven round loop ----------------------------------------------
// The counters the host round loop keeps on the host, kept on the device for
// a sort driven by a CUDA graph with conditional nodes (the graph's control
// kernels advance them and set the loops' conditions).  One per workspace.
constexpr uint32_t GRAPH_MAX_LEVELS = 4096;  // partition levels per round
constexpr uint32_t GRAPH_ROUNDS_PER_LAUNCH = 64;
constexpr uint32_t GRAPH_AUTO_MAX_N = 16u << 20;  // single sorts the auto mode runs as a graph

// Whether a round gathers its large segments' keys inside the first
// partition level's count (the rest of the sort is the same either way).
// Mode 2: always; 0: never; 1: in deep rounds (random reads, which the count
// work overlaps), and in fresh rounds of at most FUSED_FRESH_MAX keys, where
// the separate streaming gather saves less than its launches cost (measured
// on B200: 1 M keys 0.415 -> 0.394 ms per sort fused; 50 M URLs
// 9.07 -> 9.27 ms).
constexpr unsigned long long FUSED_FRESH_MAX = 1ull << 22;
__host__ __device__ inline bool gather_fused(uint32_t mode, bool fresh, unsigned long long keys) {
    return mode == 2 || (mode == 1 && (!fresh || keys <= FUSED_FRESH_MAX));
}

struct GraphState {
    uint32_t n_cur;    // segments of the current round (list R)
    uint32_t n_large;  // large segments of the current partition level (list L)
    uint32_t round;    // rounds finished in this sort
    uint32_t round_in_launch;
    uint32_t levels;   // partition levels of the current round
    uint32_t first;    // 1 while the level gathers its keys in the count kernel
    uint32_t done;     // 1 once no segment is left
    uint32_t error;    // 1: more than GRAPH_MAX_LEVELS levels in a round
    uint32_t cur_w1, cur_w8, cur_s[3], cur_e;  // on-chip sort list entries launched
    uint32_t ticket;   // CTAs finished in the current control kernel
    uint32_t fused;    // gather_fused mode (0, 1 or 2)
    uint32_t fused_round;  // 1 if the current round gathers inside its first count
    uint32_t max_levels;
    uint32_t partition_levels;
    unsigned long long small_segments, partitioned, gather_elems, gather_fused, warp1_fresh,
        warp1_keyed, warp8_fresh, warp8_keyed, block_fresh, block_keyed, equal_moved,
        equal_final, boundaries, warp1_deep, full_sorted, window_saved, window_used;
    unsigned long long live[64];
};

// ---- device workspace ---------------------------------------------------------
// Every scratch buffer of one sort of up to n strings, carved from one block
// of device memory by ws_layout (offsets, 256-byte aligned).
constexpr uint32_t SCAN_CHUNK_ELEMS = 4096;  // keys per block in the scan kernels

constexpr uint32_t scan_partials_for(uint64_t n) {
    return (uint32_t)((n ? n : 1) + SCAN_CHUNK_ELEMS - 1) / SCAN_CHUNK_ELEMS + 1;
}

struct WsLayout {
    size_t idx1, key0, key1, lcp, bkt, R, N, W1, W8, S, S2, S3, E, B, L, L2, spl, nspl, tbl, ntiles,
        cm_size, cm_base, tile_base, tmp, cm, partials, ctr, gs, lookback;
    size_t cm_cap, total;
};

constexpr WsLayout ws_layout(uint64_t n) {
    WsLayout o{};
    size_t off = 0;
    auto take = [&off](size_t bytes) {
        const size_t at = off;
        off += (bytes + 255) & ~size_t(255);
        return at;
    };
    const size_t half = n / 2 + 2;
    const size_t nlarge = n / (SMALL_CAP + 1) + 2;
    o.idx1 = take(n * 4);
    o.key0 = take(n * 16);
    o.key1 = take(n * 16);
    o.lcp = take(n * 4);
    o.bkt = take(n * 4);
    o.R = take(half * sizeof(Seg));
    o.N = take(half * sizeof(Seg));
    o.W1 = take(half * sizeof(Seg));
    o.W8 = take((n / (WARP1_CAP + 1) + 2) * sizeof(Seg));
    // class 0 starts above the one-warp cutoff, which may be lowered to 64
    o.S = take((n / 65 + 2) * sizeof(Seg));
    o.S2 = take((n / (BLOCK_CAP1 + 1) + 2) * sizeof(Seg));
    o.S3 = take((n / (BLOCK_CAP2 + 1) + 2) * sizeof(Seg));
    // equality work items: buckets of >= 2 strings, one item per EQ_TILE
    o.E = take((half + n / EQ_TILE + 2) * sizeof(Seg));
    o.B = take((n + 2) * 8);
    o.L = take(nlarge * sizeof(Seg));
    o.L2 = take(nlarge * sizeof(Seg));
    o.spl = take(nlarge * SPL_STRIDE * 16);
    o.nspl = take(nlarge * 4);
    o.tbl = take(nlarge * TBL_STRIDE * 2);
    o.ntiles = take(nlarge * 4);
    o.cm_size = take(nlarge * 4);
    o.cm_base = take((nlarge + 1) * 4);
    o.tile_base = take((nlarge + 1) * 4);
    o.tmp = take((nlarge + 1) * 4);
    // bucket-count matrix: at most NB_MAX buckets per tile of each segment
    o.cm_cap = (size_t)NB_MAX * (n / PART_TILE + nlarge + 1) + 1;
    o.cm = take(o.cm_cap * 4);
    o.partials = take((size_t)scan_partials_for(o.cm_cap) * 4);
    // single-pass scan: a ticket word, then one status word per tile
    o.lookback = take(8 + (size_t)scan_partials_for(o.cm_cap) * 8);
    o.ctr = take(sizeof(Counters));
    o.gs = take(sizeof(GraphState));
    o.total = off;
    return o;
}

struct Workspace {
    uint32_t *idx1, *lcp, *nspl, *ntiles, *cm_size, *cm_base, *tile_base, *tmp, *cm, *partials;
    unsigned char *lookback;  // ticket + tile status words of the single-pass scan
    ulonglong2 *key0, *key1, *spl;
    Seg *R, *N, *W1, *W8, *S, *S2, *S3, *E, *L, *L2;
    uint2 *B;
    uint16_t *tbl;
    uint32_t *bkt;
    Counters *ctr;
    GraphState *gs;
    size_t cm_cap;
};

inline Workspace ws_bind(const WsLayout &o, unsigned char *base) {
    Workspace w;
    w.idx1 = (uint32_t *)(base + o.idx1);
    w.key0 = (ulonglong2 *)(base + o.key0);
    w.key1 = (ulonglong2 *)(base + o.key1);
    w.lcp = (uint32_t *)(base + o.lcp);
    w.bkt = (uint32_t *)(base + o.bkt);
    w.R = (Seg *)(base + o.R);
    w.N = (Seg *)(base + o.N);
    w.W1 = (Seg *)(base + o.W1);
    w.W8 = (Seg *)(base + o.W8);
    w.S = (Seg *)(base + o.S);
    w.S2 = (Seg *)(base + o.S2);
    w.S3 = (Seg *)(base + o.S3);
    w.E = (Seg *)(base + o.E);
    w.B = (uint2 *)(base + o.B);
    w.L = (Seg *)(base + o.L);
    w.L2 = (Seg *)(base + o.L2);
    w.spl = (ulonglong2 *)(base + o.spl);
    w.nspl = (uint32_t *)(base + o.nspl);
    w.tbl = (uint16_t *)(base + o.tbl);
    w.ntiles = (uint32_t *)(base + o.ntiles);
    w.cm_size = (uint32_t *)(base + o.cm_size);
    w.cm_base = (uint32_t *)(base + o.cm_base);
    w.tile_base = (uint32_t *)(base + o.tile_base);
    w.tmp = (uint32_t *)(base + o.tmp);
    w.cm = (uint32_t *)(base + o.cm);
    w.partials = (uint32_t *)(base + o.partials);
    w.lookback = base + o.lookback;
    w.ctr = (Counters *)(base + o.ctr);
    w.gs = (GraphState *)(base + o.gs);
    w.cm_cap = o.cm_cap;
    return w;
}

// ---- launchers (ssort_kernels.cu) ----------------------------------------
void launch_iota(uint32_t *idx, uint32_t n, cudaStream_t st);
// 256-bin histogram of the first 8 key bytes of `samples` strings (tuning).
void launch_byte_hist(const uint8_t *arena, uint64_t arena_bytes, const void *offs, int off_width,
                      uint32_t n, uint32_t samples, uint32_t *hist, cudaStream_t st);
// Launchers with a Count take `grid` CTAs (or size the grid from a host count
// when grid <= 0); their kernels loop over the work they find.
void launch_classify(const Seg *R, Count nR, uint32_t warp8_cap, Seg *W1, Seg *W8,
                     SmallLists S, Seg *L, Counters *c, int grid, cudaStream_t st);
// Batches: one round-0 segment per instance; instance-local result indices.
void launch_init_batch(const uint32_t *inst_start, uint32_t ninst, Seg *R, uint32_t *lcp,
                       Counters *c, cudaStream_t st);
uint64_t text_tiles(uint64_t len);  // CTAs (tile counts) of the text kernels
void launch_text_count(const uint8_t *text, uint64_t len, uint8_t delim, uint32_t *tile_cnt,
                       unsigned long long *total, cudaStream_t st);
void launch_text_starts(uint8_t *text, uint64_t len, uint8_t delim, const uint32_t *tile_base,
                        uint64_t n, void *offs, int off_width, cudaStream_t st);
void launch_iota_offs(void *offs, int off_width, uint64_t n, cudaStream_t st);
void launch_sorted_offs(const uint32_t *perm, const void *offs, int off_width, uint64_t n,
                        void *out, int out_width, cudaStream_t st);
// One request joining or leaving the server's batch (see k_join / k_unbase).
struct ReqJob {
    uint64_t region_base, arena_bytes;
    uint32_t pos, n;
    uint32_t first;  // positions of the jobs before this one
    uint32_t slot;   // segment slot in the round list (requests of >= 2 strings)
    uint32_t off_width, pad;
};
void launch_join(uint64_t *goffs, uint32_t *lcp, uint32_t *perm, const ReqJob *jobs,
                 uint32_t njobs, uint32_t total, Seg *R, cudaStream_t st);
void launch_mark(const Seg *R, uint32_t nR, const uint32_t *base, uint32_t nact, uint32_t *flag,
                 cudaStream_t st);
void launch_unbase(uint32_t *perm, const ReqJob *jobs, uint32_t njobs, uint32_t total,
                   cudaStream_t st);
void launch_localize(uint32_t *perm, uint32_t n, const uint32_t *inst_start, uint32_t ninst,
                     cudaStream_t st);
// Single-CTA scans of short per-segment arrays (out*[n] = totals).
void launch_scan_pair(const uint32_t *in0, uint32_t *out0, const uint32_t *in1, uint32_t *out1,
                      Count n, cudaStream_t st);
void launch_seg_tiles(const Seg *segs, Count n, uint32_t tile, uint32_t *out, cudaStream_t st);
// exclusive scan of in[0..n) into out[0..n); out[n] = total (out has n+1 slots).
// cap (host) bounds n and sizes the grid; n itself is count_of(n).
void launch_scan(const uint32_t *in, uint32_t *out, uint32_t cap, Count n, uint32_t *partials,
                 cudaStream_t st);
uint32_t scan_partials_needed(uint32_t n);
// The same scan in one pass with decoupled look-back: tiles take their order
// from a ticket and add up their predecessors' published sums; `state` holds
// a ticket word and one status word per tile and must be zeroed first
// (lookback_state_bytes(cap)); a look-back that waits too long sets *err.
size_t lookback_state_bytes(uint32_t cap);
void launch_scan_lookback(const uint32_t *in, uint32_t *out, uint32_t cap, Count n,
                          unsigned char *state, uint32_t *err, cudaStream_t st);
void launch_gather(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                   Counters *c, int grid, cudaStream_t st);
// from_arena / gather: first partition level of a round, whose keys the
// count kernel gathers from the arena (the sample reads its strings there).
void launch_sample(const SortArgs &a, const Seg *L, Count nL, ulonglong2 *spl,
                   uint32_t *nspl, uint16_t *tbl, uint32_t *ntiles, uint32_t *cm_size,
                   bool from_arena, int grid, cudaStream_t st);
void launch_count(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                  const ulonglong2 *spl, const uint32_t *nspl, const uint16_t *tbl,
                  const uint32_t *cm_base, uint32_t *cm, Counters *c, bool gather, int grid,
                  cudaStream_t st);
void launch_scatter(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                    const ulonglong2 *spl, const uint32_t *nspl, const uint16_t *tbl,
                    const uint32_t *cm_base, const uint32_t *cm_scan, int grid,
                    cudaStream_t st);
void launch_emit(const SortArgs &a, const Seg *L, Count nL, const uint32_t *tile_base,
                 const uint32_t *nspl, const uint32_t *cm_base, const uint32_t *cm_scan,
                 Seg *W1, Seg *W8, SmallLists S, Seg *L2, Seg *E, uint2 *B, Seg *N,
                 Counters *c, int grid, cudaStream_t st);
// On-chip segment sorts; list lengths are read from the counters on the device.
// The on-chip sorts take n list entries from the given list pointer (a range
// of the list), so that they can run while the list is still being appended.
void launch_warp1(const SortArgs &a, const Seg *W1, Span sp, Seg *N, Counters *c, int grid,
                  cudaStream_t st);
void launch_warp8(const SortArgs &a, const Seg *W8, Span sp, Seg *N, Counters *c, int grid,
                  cudaStream_t st);
// cls: size class 0, 1, 2 (segment list S holds that class)
// prefetch: the double-buffered variant (records of the next segment copied
// asynchronously while the current one sorts; two CTAs per SM instead of three).
void launch_block(const SortArgs &a, const Seg *S, Span sp, int cls, Seg *N, Counters *c,
                  int grid, cudaStream_t st, bool prefetch);
void launch_equal(const SortArgs &a, const Seg *E, Span sp, Seg *N, Counters *c, int grid,
                  cudaStream_t st);
void launch_boundary(const SortArgs &a, const uint2 *B, Counters *c, int grid, cudaStream_t st);

// Control kernels of the device-driven round loop.  Conditions are
// cudaGraphConditionalHandle values (unsigned long long).
// Round start: clear the round's counters and the sort-list cursors (and the
// round condition, which only the round's last kernel sets again).
void launch_g_round_begin(GraphState *g, Counters *c, unsigned long long h_round,
                          cudaStream_t st);
// After classification: the level loop's condition (large segments left) and
// whether this round gathers its keys with a separate pass (round 0, or the
// fused gather switched off).
void launch_g_after_classify(GraphState *g, Counters *c, unsigned long long h_level,
                             unsigned long long h_gather, cudaStream_t st);
// Before a level: whether its count kernel gathers the keys itself (and the
// level condition cleared, set again only by the level's last kernel).
void launch_g_level_begin(GraphState *g, unsigned long long h_level, unsigned long long h_first,
                          cudaStream_t st);
// After a level: the next level's large segments move from L2 to L, the
// cursors advance past the on-chip sorts launched, the level condition is set.
void launch_g_level_end(GraphState *g, Counters *c, Seg *L, const Seg *L2,
                        unsigned long long h_level, int grid, cudaStream_t st);
// After a round: its statistics are added up, the next round's segments move
// from N to R, and the round condition is set.
void launch_g_round_end(GraphState *g, Counters *c, Seg *R, const Seg *N,
                        unsigned long long h_round, int grid, cudaStream_t st);

}  // namespace ssort
