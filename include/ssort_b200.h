/*
 * ssort_b200.h -- C ABI of the B200 MSD radix string sort (libssort_b200.so).
 *
 * Plain C: pointers, sizes and status codes only.  Every entry point that can
 * fail returns an int status (SSORT_OK = 0, negative on error); the drop-in
 * routine msd_gpu follows the reference's convention instead and aborts with
 * a message, since struct routine::f has no return value.
 *
 * Sort contract (all entry points): the output order is the stable byte-order
 * sort of the NUL-terminated strings, i.e. the order the reference's msd_CE6
 * produces (rantala/string-sorting src/msd_ce.cpp:367-419; stable because its
 * counting sort is, :396-397, and its insertion sort breaks ties on <=,
 * src/util/insertion_sort.h:42).  Bytes compare as unsigned char.
 * perm[k] is the input index of the k-th string in that order.  The LCP array
 * uses the reference's lcp() (src/mergesort_lcp.cpp:88-100): lcp[0] = 0 and
 * lcp[k] = number of equal leading bytes of strings perm[k-1] and perm[k],
 * stopping at the first difference or at the NUL of the first string.
 */
#ifndef SSORT_B200_H
#define SSORT_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SSORT_OK 0
#define SSORT_EINVAL (-1)    /* bad argument (null pointer, bad width, n too big) */
#define SSORT_ENOMEM (-2)    /* device or pinned host allocation failed */
#define SSORT_ECUDA (-3)     /* a CUDA runtime call failed */
#define SSORT_ENODEV (-4)    /* no usable CUDA device */
#define SSORT_EINTERNAL (-5) /* an internal consistency check failed */

/* Largest number of strings one sort accepts (indices are 32-bit). */
#define SSORT_MAX_N 0xFFFFFFFEull
#define SSORT_MAX_ROUNDS 64

typedef struct ssort_ctx ssort_ctx;

/*
 * Drop-in routine.  Same signature and contract as the reference's
 * struct routine::f (src/routine.h:32-37), registered through
 * ROUTINE_REGISTER_SINGLECORE(msd_gpu, ...) (src/routine.h:55-56) exactly
 * where msd_CE6 registers (src/msd_ce.cpp:418-419).  Permutes strings[0..n)
 * in place into stable byte order; never touches the string bytes.  Works on
 * any pointers (one text buffer as in sortstring, or separately allocated
 * strings as in unit-test/main.cpp:220-270).  Uses one process-wide context
 * on the current CUDA device.  Aborts with a message on any CUDA error (the
 * reference's convention, src/routines.c:33-40); there is no CPU fallback.
 */
void msd_gpu(unsigned char **strings, size_t n);

/* Human-readable name of a status code, and the message of the last error
 * raised on the calling thread. */
const char *ssort_strerror(int status);
const char *ssort_last_error(void);

/* A context owns a CUDA stream and the device workspace; workspaces grow on
 * demand and are reused across calls.  One context must not be used by two
 * threads at once; separate contexts are independent. */
int ssort_ctx_create(int device, ssort_ctx **out);
void ssort_ctx_destroy(ssort_ctx *ctx);

/*
 * Device-resident sort: d_arena holds the strings (16-byte aligned base
 * address, arena_bytes long), d_offs holds n offsets of width off_width
 * (4 or 8 bytes; string i starts at d_arena + d_offs[i] and is NUL-terminated
 * inside the arena).  Writes d_perm[n] and, if d_lcp is not NULL, d_lcp[n].
 * `stream` is a cudaStream_t (NULL = the context's own stream).  Returns when
 * the results are complete on the device.
 */
int ssort_sort_device(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                      const void *d_offs, int off_width, uint64_t n, uint32_t *d_perm,
                      uint32_t *d_lcp, void *stream);

/*
 * ssort_sort_device without any device allocation.  This entry point has no
 * counterpart in the reference; it exists for callers that cannot let a
 * library allocate device memory: cudaMalloc/cudaFree synchronise the device
 * and can fail when the application has already budgeted all memory to its
 * own pool.  All scratch lives in one fixed device array inside the library
 * (SSORT_NOALLOC_MAX_N strings' worth, about 24 MB), which every GPU that
 * loads the library holds until the process exits; larger n is rejected with
 * SSORT_EINVAL.  The caller still passes the inputs and the perm (and
 * optional lcp) outputs, and a cudaStream_t (NULL = the legacy default
 * stream); the call waits for that stream (cudaStreamSynchronize) before it
 * returns, on failure too, so the results are complete.  Because of that
 * wait, and the host reads of counters between kernels, it must not be called
 * while its stream (or, for its first call on a device, which looks up the
 * array's address with cudaGetSymbolAddress, any stream) is being captured
 * into a CUDA graph.  Every call uses the same array
 * and leaves its contents behind (what must start at zero is cleared by each
 * call).  Calls that overlapped on the GPU would race on the array; the
 * library prevents that within one process by taking a lock for the whole
 * call and returning only after the call's GPU work has finished.
 */
#define SSORT_NOALLOC_MAX_N 262144u
int ssort_sort_device_noalloc(const uint8_t *d_arena, uint64_t arena_bytes, const void *d_offs,
                              int off_width, uint64_t n, uint32_t *d_perm, uint32_t *d_lcp,
                              void *stream);

/* The same from host buffers: copies arena and offsets to the device, sorts,
 * and copies perm (and lcp when not NULL) back.  Pinned host buffers make the
 * copies faster but are not required.  With off_width 8, an arena below 4 GB
 * and n >= 2^20, the offsets are narrowed to 4 bytes on the host (into a
 * pinned buffer the context keeps) while the arena is being copied, and only
 * those cross to the device; the caller's buffers are only read. */
int ssort_sort_host(ssort_ctx *ctx, const uint8_t *arena, uint64_t arena_bytes,
                    const void *offs, int off_width, uint64_t n, uint32_t *perm,
                    uint32_t *lcp);

/*
 * Batched sort: ninst independent instances in one call (no counterpart in
 * the reference, which sorts one array per call).  Instance i owns positions
 * inst_start[i] .. inst_start[i+1]-1 of the offsets array (inst_start has
 * ninst + 1 non-decreasing entries, inst_start[0] = 0, inst_start[ninst] = n);
 * its strings may live anywhere in the shared arena.  For a position p of
 * instance i, perm[p] is the index, counted from inst_start[i], of the string
 * of instance i ranked p - inst_start[i]; lcp restarts at 0 for every
 * instance.  All instances are refined together: every kernel launch works
 * on the live segments of all of them.
 */
int ssort_sort_batch_device(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                            const void *d_offs, int off_width, uint64_t n,
                            const uint32_t *d_inst_start, uint32_t ninst, uint32_t *d_perm,
                            uint32_t *d_lcp, void *stream);
int ssort_sort_batch_host(ssort_ctx *ctx, const uint8_t *arena, uint64_t arena_bytes,
                          const void *offs, int off_width, uint64_t n, const uint32_t *inst_start,
                          uint32_t ninst, uint32_t *perm, uint32_t *lcp);

/* Pointer-array form behind msd_gpu with a status return: permutes
 * strings[0..n) in place and, when lcp_out is not NULL, writes the LCP array
 * of the sorted order. */
int ssort_sort_strings(ssort_ctx *ctx, unsigned char **strings, size_t n, uint32_t *lcp_out);

/*
 * Text inputs: the strings of a whole input file, as the reference's
 * sortstring makes them (src/sortstring.c:310-358), found on the GPU instead
 * of by a host pass that builds a pointer array.
 *   SSORT_TEXT_LINES     every '\n' ends a string and becomes its NUL
 *                        (create_strings_delim with '\n', the default mode);
 *   SSORT_TEXT_RAW       every NUL ends a string (--raw);
 *   SSORT_TEXT_SUFFIXES  every position starts a string: all suffixes of the
 *                        text (--suffix-sorting, create_suffixes).
 * In the delimited modes the string after the last delimiter is not a string
 * (as in the reference).  Bytes at or past text_len read as NUL.
 *
 * ssort_text_offsets_device writes the string starts into d_offs (width 4 or
 * 8; width 4 needs text_len < 2^32) on `stream` and returns their number in
 * *n_out.  With SSORT_TEXT_LINES it overwrites the '\n' bytes of d_text with
 * NUL.  When the strings would exceed cap entries it writes nothing, sets
 * *n_out to the number needed and returns SSORT_EINVAL.
 *
 * ssort_sort_text_host sorts the strings of a host text: sorted_offs[k] is the
 * start (offset into text) of the k-th smallest string; lcp (optional) as for
 * every sort.  Capacity and *n_out as above.  The host text is not modified.
 */
#define SSORT_TEXT_LINES 0
#define SSORT_TEXT_RAW 1
#define SSORT_TEXT_SUFFIXES 2
int ssort_text_offsets_device(ssort_ctx *ctx, uint8_t *d_text, uint64_t text_len, int mode,
                              void *d_offs, int off_width, uint64_t cap, uint64_t *n_out,
                              void *stream);
int ssort_sort_text_host(ssort_ctx *ctx, const uint8_t *text, uint64_t text_len, int mode,
                         uint64_t *sorted_offs, uint32_t *lcp, uint64_t cap, uint64_t *n_out);

/*
 * LCP consumers (no counterpart entry point in the reference; the merge is its
 * mergesort_lcp two-way LCP merge, src/mergesort_lcp.cpp:133-211).
 *
 * ssort_merge_runs merges sorted runs on the host using their LCP arrays.
 * Run r owns positions run_start[r] .. run_start[r+1]-1 (run_start has
 * nruns + 1 non-decreasing entries from 0 to n); perm/lcp hold each run's
 * result as the batched sort returns it (indices local to the run, lcp
 * restarting at 0).  Writes the global order (indices into offs) and its LCP
 * array: exactly the sort of all n strings in one call.  The outputs may
 * alias the inputs.  Runs with OpenMP threads.
 *
 * ssort_sort_host_chunked sorts n strings with a device workspace sized for
 * chunk_strings only: the arena is copied once, consecutive chunks of
 * chunk_strings offsets are sorted on the GPU one after another, and the runs
 * are merged with ssort_merge_runs.  Results as ssort_sort_host.
 */
int ssort_merge_runs(const uint8_t *arena, uint64_t arena_bytes, const void *offs,
                     int off_width, uint64_t n, const uint32_t *run_start, uint32_t nruns,
                     const uint32_t *perm, const uint32_t *lcp, uint32_t *out_perm,
                     uint32_t *out_lcp);
int ssort_sort_host_chunked(ssort_ctx *ctx, const uint8_t *arena, uint64_t arena_bytes,
                            const void *offs, int off_width, uint64_t n, uint64_t chunk_strings,
                            uint32_t *perm, uint32_t *lcp);

/* Page-locked host memory (for reading inputs straight into a buffer that the
 * copy engines read at full speed); freed with ssort_pinned_free. */
int ssort_pinned_alloc(size_t bytes, void **out);
void ssort_pinned_free(void *p);

/* Per-call statistics of the last sort on this context. */
typedef struct {
    uint64_t n;                              /* strings sorted */
    uint32_t rounds;                         /* 16-byte refinement rounds run */
    uint32_t partition_levels;               /* sample-partition passes run */
    uint64_t live[SSORT_MAX_ROUNDS];         /* strings live entering each round */
    uint64_t partitioned;                    /* elements moved by partition scatters */
    uint64_t small_segments;                 /* segments sorted on chip */
    uint64_t device_bytes;                   /* device workspace currently held */
    double device_ms;                        /* device time of the sort (events) */
    /* strings handled per kernel, summed over rounds: keys gathered for large
     * segments; strings sorted by the one-per-lane warp sort, the
     * eight-per-lane warp sort and the CTA sort, with keys loaded in the
     * kernel ("fresh") or taken from the key buffer ("keyed"); equality-bucket
     * strings moved between buffers / finalised; partition boundaries. */
    uint64_t gather_elems;
    uint64_t warp1_fresh, warp1_keyed, warp8_fresh, warp8_keyed, block_fresh, block_keyed;
    uint64_t equal_moved, equal_final;
    uint64_t boundaries;
    uint64_t gather_fused; /* of gather_elems: keys gathered by the first
                              partition level's count kernel (rounds >= 1) */
    uint64_t warp1_deep;   /* strings re-sorted by the one-per-lane warp sort on
                              their next 16 bytes within the same round
                              (SSORT_PARAM_WARP1_DEEP), summed over steps */
    uint64_t full_sorted;  /* strings of on-chip sorted segments whose packed
                              64-bit keys could not order them (a run of more
                              than 64 equal windows) and were re-sorted with
                              the full key comparator */
    uint64_t window_saved; /* strings whose key bytes 16..31 round 0's gather
                              kept for round 1 (sorts of at least 2^20 strings
                              whose arena holds >= 24 bytes per string, unless
                              the context's previous sort sent fewer than a
                              quarter of its strings into round 1) */
    uint64_t window_used;  /* round-1 keys read from those copies instead of
                              through the offset and the arena */
    uint64_t graph_launches; /* launches of the device-driven loop's graph
                                (0: the host drove the rounds) */
} ssort_stats;

int ssort_get_stats(const ssort_ctx *ctx, ssort_stats *out);

/* Tuning parameters of a context (defaults are chosen per size class inside
 * the library; these override them for every later sort on the context). */
#define SSORT_PARAM_TARGET_BUCKET 1 /* wanted strings per range bucket of a sample
                                       partition, 32..2048 (default 512) */
#define SSORT_PARAM_WARP8_CAP 2     /* largest segment sorted by one warp, 64..256
                                       (default 256); larger ones go to the CTA sort */
#define SSORT_PARAM_OVERLAP 3       /* 1 (default): in every round the on-chip sorts run
                                       on a side stream beside the partition; 0: one stream */
#define SSORT_PARAM_FUSED_GATHER 4  /* 1 (default): the first partition level of a
                                       round gathers the keys it counts, except in a round 0
                                       of more than 4 M keys, which streams them in a
                                       separate pass first; 2: every round; 0: separate
                                       gather in every round */
#define SSORT_PARAM_WARP1_DEEP 5    /* 0..4096 (default 64): 16-byte steps the warp that
                                       sorts a segment of <= 32 strings takes on its own
                                       runs of equal keys before handing what is left to
                                       the next round; 0: every run waits for the next round */
#define SSORT_PARAM_BLOCK_PREFETCH 6 /* 0 (default): the CTA sort of segments of 257..2048
                                        strings loads one segment's records through
                                        registers at three CTAs per SM; 1: it copies the
                                        next segment's records into shared memory while it
                                        sorts the current one (two CTAs per SM) */
#define SSORT_PARAM_MATCH_VOTE 13    /* 1: the partition's count kernel finds the lanes of a
                                        warp that share a bucket with one ballot per
                                        bucket-id bit; 0 (default): with __match_any_sync */
#define SSORT_PARAM_SCAN 15          /* 1 (default): the partition's count-matrix scan runs
                                        in one pass with decoupled look-back (tiles in
                                        ticket order add up their predecessors' published
                                        sums); 0: reduce, scan of the partials, down-sweep */
#define SSORT_PARAM_WARP_MERGE 14    /* 1 (default): the warp-level sorts of packed keys
                                        (one-warp and CTA sorts) sort each lane's values
                                        with a sorting network and merge runs with
                                        merge-path passes; 0: a bitonic network across
                                        the warp */
#define SSORT_PARAM_BLOCK_LEAN 12    /* 1: the CTA sort takes the LCPs of neighbours whose
                                        packed windows differ from the windows alone and
                                        reads full keys only for equal windows; 2: that, and
                                        its first sort runs on 32-bit packed keys (21 key
                                        bits and the position; ties on those bits are put in
                                        order afterwards); 0 (default): full-key finish */
#define SSORT_PARAM_L2_PREFETCH 9    /* 1: the partition's count and scatter kernels ask
                                        for their next tile to be streamed into L2 (bulk
                                        prefetch) while they work on the current one;
                                        0 (default): no such requests */
#define SSORT_PARAM_DIGIT_BITS 10    /* 8, 9 or 10 (default 10): digit width of one
                                        partition pass, i.e. a pass splits a segment into
                                        at most 2^bits buckets (2^(bits-1) - 1 sampled
                                        splitters and the buckets between and at them) */
#define SSORT_PARAM_SCATTER 11       /* 0 (default): the partition scatter lays each tile out
                                        in shared memory in output order; 1: it stages only
                                        indices and destinations and reads each key from the
                                        tile (in L2) in output order, at more CTAs per SM;
                                        2: as 0, with each bucket run of keys written by one
                                        asynchronous bulk copy from shared memory */
#define SSORT_PARAM_GRAPH 7          /* 1: device-driven round loop: the sort runs as a CUDA
                                        graph whose rounds and partition levels are
                                        conditional loops (no host round trip between
                                        kernels; one host read per up to 64 rounds);
                                        0 (default): the host drives the rounds; 2: the
                                        graph for batched sorts and sorts of at most 2^24
                                        strings, from the second of two sorts in a row with
                                        the same buffers and size on (building a graph
                                        costs more than a host-driven sort) */
#define SSORT_PARAM_GRAPH_MAX_LEVELS 8 /* 1..4096 (default 4096): partition levels one round
                                          of the device-driven loop may take; a round that
                                          needs more fails with SSORT_EINTERNAL */
int ssort_set_param(ssort_ctx *ctx, int param, int64_t value);

/*
 * Autotuning (no counterpart in the reference).  Times sorts of the given
 * device input under candidate parameter values, one parameter at a time:
 * target bucket {256, 512, 1024}, one-warp cutoff {64, 128, 256}, fused
 * gather {1, 0}, overlap {1, 0}; each candidate is sorted twice and kept when
 * its faster run beats the current best by at least 1 %.  The winners are
 * set on the context and recorded for the input's size class (floor(log2 n))
 * and entropy class (Shannon entropy of the first 8 key bytes of a 4096-string
 * sample: < 2, < 4, >= 4 bits per byte); later sorts on this context whose
 * input falls in a recorded class use that class's values (when a size class
 * has values for more than one entropy class, one sample pass finds the
 * class).  Results are identical under every parameter value.
 */
typedef struct {
    uint32_t size_class;    /* floor(log2 n) */
    uint32_t entropy_class; /* 0, 1, 2 (see above) */
    double entropy_bits;    /* bits per byte of the sample */
    int64_t target_bucket, warp8_cap, overlap, fused_gather; /* chosen values */
    double default_ms;      /* device time of one sort with the values before tuning */
    double tuned_ms;        /* with the chosen values */
    uint32_t trials;        /* sorts timed */
    int64_t digit_bits, block_prefetch, l2_prefetch, graph; /* chosen values */
} ssort_tuning;
int ssort_autotune(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                   const void *d_offs, int off_width, uint64_t n, ssort_tuning *out);

/* Kernel-level timing: when enabled, each kernel launch of a sort is bracketed
 * by CUDA events and its time is accumulated per kernel name. */
int ssort_set_profiling(ssort_ctx *ctx, int enabled);
/* Fills up to max entries; returns the number of distinct kernels recorded. */
int ssort_get_kernel_times(const ssort_ctx *ctx, const char **names, double *total_ms,
                           uint64_t *launches, int max);

/* ---- request server (continuous batching) ----------------------------------
 * No reference counterpart: the reference sorts one pointer array per call.
 * A server owns one device: a pool arena of arena_budget_bytes for the
 * strings of admitted requests and per-string state for max_strings
 * positions.  Requests are submitted from host buffers and queued; each
 * ssort_server_step admits queued requests in FIFO order while their bytes
 * (arena_bytes + 1, rounded up to 256) and strings fit the free pool and
 * position ranges, starts their copies on a copy stream, joins the requests
 * whose copies have landed into the running segment list as depth-0
 * segments, runs ONE refinement round over the segments of every joined
 * request together, and starts the device-to-host copy of each request that
 * has no segment left.  Requests therefore enter and leave the batch between
 * rounds.  Each result is exactly what ssort_sort_host returns for the same
 * request alone: perm local to the request, lcp[0] = 0.
 *
 * The caller's arena, offs, perm_out and lcp_out may be host memory or
 * device memory of the server's device (copies use unified addressing); they
 * must stay valid and the inputs unmodified until the request is reported
 * done.  Pinned host memory lets host copies overlap the rounds.  A server is not shared between
 * threads without outside locking; every call takes its lock. */
typedef struct ssort_server ssort_server;

#define SSORT_REQ_QUEUED 0   /* submitted, waiting for pool space */
#define SSORT_REQ_LOADING 1  /* admitted, host-to-device copy in flight */
#define SSORT_REQ_ACTIVE 2   /* segments in the running batch */
#define SSORT_REQ_DRAINING 3 /* sorted, device-to-host copy in flight */
#define SSORT_REQ_DONE 4     /* perm_out / lcp_out written */

typedef struct {
    uint32_t queued, loading, active, draining; /* requests per state */
    uint32_t max_active;                        /* most requests joined at once */
    uint64_t rounds;                            /* rounds run */
    uint64_t requests_done, strings_done;       /* completed so far */
    uint64_t arena_in_use, strings_in_use;      /* pool bytes / positions held */
    uint64_t arena_budget, max_strings;         /* capacities */
    uint64_t device_bytes;                      /* device memory held */
} ssort_server_info;

int ssort_server_create(int device, uint64_t arena_budget_bytes, uint64_t max_strings,
                        ssort_server **out);
void ssort_server_destroy(ssort_server *srv);
/* Queues one request (n strings at arena + offs[i], offsets of off_width 4 or
 * 8 bytes).  SSORT_ENOMEM when it could never fit the server's capacities.
 * lcp_out may be NULL.  n == 0 completes at once. */
int ssort_server_submit(ssort_server *srv, const uint8_t *arena, uint64_t arena_bytes,
                        const void *offs, int off_width, uint64_t n, uint32_t *perm_out,
                        uint32_t *lcp_out, uint64_t *id_out);
/* One scheduling step (see above).  Writes up to cap ids of requests that
 * completed since the last report into done_ids and their count into *n_done;
 * the rest are reported by later steps. */
int ssort_server_step(ssort_server *srv, uint64_t *done_ids, uint32_t cap, uint32_t *n_done);
/* State (SSORT_REQ_*) of request id. */
int ssort_server_poll(ssort_server *srv, uint64_t id, int *state);
/* Steps until every submitted request is done; completions are still
 * reported by the next ssort_server_step calls. */
int ssort_server_drain(ssort_server *srv);
int ssort_server_get_info(ssort_server *srv, ssort_server_info *out);

#ifdef __cplusplus
}
#endif

#endif /* SSORT_B200_H */
