// ssort_engine.cu -- host side of the B200 MSD radix string sort: the context
// and its device workspace, the round loop that drives the kernels, and the
// C ABI declared in include/ssort_b200.h (including the drop-in routine
// msd_gpu that registers through the reference's ROUTINE_REGISTER,
// src/routine.h:41-59).
#include "ssort_host.cuh"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>
#include <omp.h>

using namespace ssort;

namespace {
thread_local std::string g_last_error;
}  // namespace

int ssort::fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int ssort::cuda_fail(cudaError_t e, const char *what) {
    return fail(SSORT_ECUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int ssort_ctx::reserve(uint32_t n) {
    if (ws_buf.p && n <= ws_n) return SSORT_OK;
    const WsLayout lay = ws_layout(n);
    SS_TRY(ensure(ws_buf, lay.total));
    ws = ws_bind(lay, (unsigned char *)ws_buf.p);
    ws_n = n;
    if (!h_ctr) {
        SS_CUDA(cudaHostAlloc((void **)&h_ctr, sizeof(Counters), cudaHostAllocDefault));
    }
    return SSORT_OK;
}

// Shannon entropy (bits per byte) of the first 8 key bytes of up to 4096
// strings spread over the input.
int ssort_ctx::sample_entropy(const uint8_t *arena_p, uint64_t arena_bytes, const void *offs_p,
                              int off_width, uint32_t n, double &bits) {
    SS_TRY(ensure(hist_buf, 256 * 4));
    if (!h_hist) SS_CUDA(cudaHostAlloc((void **)&h_hist, 256 * 4, cudaHostAllocDefault));
    const uint32_t samples = std::min<uint32_t>(n, 4096);
    LAUNCH(this, "byte_hist",
           launch_byte_hist(arena_p, arena_bytes, offs_p, off_width, n, samples,
                            (uint32_t *)hist_buf.p, st));
    SS_CUDA(cudaMemcpyAsync(h_hist, hist_buf.p, 256 * 4, cudaMemcpyDeviceToHost, st));
    SS_CUDA(cudaStreamSynchronize(st));
    double total = 0, h = 0;
    for (int b = 0; b < 256; ++b) total += h_hist[b];
    for (int b = 0; b < 256; ++b)
        if (h_hist[b]) {
            const double p = h_hist[b] / total;
            h -= p * std::log2(p);
        }
    bits = h;
    return SSORT_OK;
}

int ssort_ctx::scan(const uint32_t *in, uint32_t *out, uint32_t cap, Count n) {
    return scan_on(in, out, cap, n, st);
}

// The count-matrix scan on stream s: single-pass with decoupled look-back
// (SSORT_PARAM_SCAN = 1; its state is cleared first), or reduce-then-scan.
int ssort_ctx::scan_on(const uint32_t *in, uint32_t *out, uint32_t cap, Count n,
                       cudaStream_t s) {
    if (scan_lookback) {
        SS_CUDA(cudaMemsetAsync(ws.lookback, 0, lookback_state_bytes(cap), s));
        LAUNCH(this, "scan",
               launch_scan_lookback(in, out, cap, n, ws.lookback, &ws.ctr->error, s));
    } else {
        LAUNCH(this, "scan", launch_scan(in, out, cap, n, ws.partials, s));
    }
    return SSORT_OK;
}

// Marks, on the partition stream, the point after which the list entries
// counted in h_ctr are ready for the on-chip sorts.
int ssort_ctx::fork_small() {
    if (overlap_round) SS_CUDA(cudaEventRecord(ev_fork, st));
    return SSORT_OK;
}

// Launches the on-chip sorts (warp, CTA and equality-bucket work) for the
// list entries appended since the last call, as counted in h_ctr.  They work
// on positions that no later partition level of the round touches, and they
// append next-round segments with atomics, so they may run concurrently with
// the partition levels on the side stream.
int ssort_ctx::launch_small(const SortArgs &a, Seg *nxt, SmallDone &d) {
    const bool overlap = overlap_round;
    // The warp and equality-bucket work on `side`, the CTA sorts on `side2`:
    // disjoint segments, so the two also run beside each other.
    cudaStream_t s2 = overlap ? side : st, s3 = overlap ? side2 : st;
    if (overlap) {
        SS_CUDA(cudaStreamWaitEvent(side, ev_fork, 0));  // recorded by fork_small
        SS_CUDA(cudaStreamWaitEvent(side2, ev_fork, 0));
    }
    Counters *dc = ws.ctr;
    // One pass of CTAs over the entries (no CTA loops over several): short
    // CTAs let the scheduler give SMs back to the partition kernels.  The
    // packed warp sort keeps a capped grid: its warps loop over entries.
    auto grid = [&](uint32_t n, uint32_t per_cta) { return (int)((n + per_cta - 1) / per_cta); };
    uint32_t n = h_ctr->n_w1 - d.w1;
    LAUNCH(this, "warp1",
           launch_warp1(a, ws.W1, hspan(d.w1, d.w1 + n), nxt, dc,
                        std::min(grid(n, 32), grid_for(8)), s2));
    d.w1 += n;
    n = h_ctr->n_w8 - d.w8;
    LAUNCH(this, "warp8", launch_warp8(a, ws.W8, hspan(d.w8, d.w8 + n), nxt, dc, grid(n, 8), s2));
    d.w8 += n;
    // CTA-sort size classes: groups of 64, 128, 256 threads per segment.
    Seg *lists[3] = {ws.S, ws.S2, ws.S3};
    const uint32_t counts[3] = {h_ctr->n_small, h_ctr->n_small2, h_ctr->n_small3};
    for (int k = 0; k < 3; ++k) {
        n = counts[k] - d.s[k];
        const uint32_t per_cta = (uint32_t)SMALL_THREADS / (64u << k);
        LAUNCH(this, "block",
               launch_block(a, lists[k], hspan(d.s[k], d.s[k] + n), k, nxt, dc,
                            grid(n, per_cta * (block_prefetch ? 4u : 1u)), s3, block_prefetch));
        d.s[k] += n;
    }
    n = h_ctr->n_equal - d.e;
    LAUNCH(this, "equal", launch_equal(a, ws.E, hspan(d.e, d.e + n), nxt, dc, grid(n, 1), s2));
    d.e += n;
    return SSORT_OK;
}

// One refinement round over the n_cur segments in `cur`: classification,
// key gather and sample partitioning of large segments, on-chip sorts,
// equality buckets and boundary LCPs.  The next round's segments are
// appended to `nxt`; their count is returned in n_next.
int ssort_ctx::round(const SortArgs &a, Seg *cur, uint32_t n_cur, Seg *nxt, uint32_t &n_next,
                     uint32_t round_no) {
    // A fresh round (round 0 of a sort, or by the caller's choice) streams
    // the arena in index order with a separate gather; a deep round gathers
    // keys at random inside the first count.  Every round overlaps its
    // on-chip sorts with its partition levels (a side stream), unless
    // switched off or timing kernels one by one.
    fresh_round = round_mode >= 0 ? round_mode == 0 : round_no == 0;
    overlap_round = side && side2 && hp && !prof && overlap;
    if (!overlap_round) return round_body(a, cur, n_cur, nxt, n_next, round_no);
    // Fork the round onto the high-priority stream and join it back.
    cudaStream_t user = st;
    SS_CUDA(cudaEventRecord(ev_round, user));
    SS_CUDA(cudaStreamWaitEvent(hp, ev_round, 0));
    st = hp;
    const int rc = round_body(a, cur, n_cur, nxt, n_next, round_no);
    st = user;
    if (rc != SSORT_OK) return rc;
    SS_CUDA(cudaEventRecord(ev_round, hp));
    SS_CUDA(cudaStreamWaitEvent(user, ev_round, 0));
    return SSORT_OK;
}

int ssort_ctx::round_body(const SortArgs &a, Seg *cur, uint32_t n_cur, Seg *nxt,
                          uint32_t &n_next, uint32_t round_no) {
    Counters *dc = ws.ctr;
    const int g8 = grid_for(8), g4 = grid_for(4), g2 = grid_for(2);
    SS_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), st));
    LAUNCH(this, "classify",
           launch_classify(cur, hcount(n_cur), a.warp8_cap, ws.W1, ws.W8,
                           SmallLists{{ws.S, ws.S2, ws.S3}}, ws.L, dc, 0, st));
    SS_TRY(sync_counters());
    if (round_no < SSORT_MAX_ROUNDS) stats.live[round_no] = h_ctr->live_next;
    // The on-chip sorts of the segments known after each host read of the
    // counters are launched on the side stream after the next partition
    // level is enqueued, so that the level's kernels get the SMs first.
    SmallDone done;
    SS_TRY(fork_small());
    uint32_t n_large = h_ctr->n_large;
    Seg *lcur = ws.L, *lnext = ws.L2;
    // Keys of the large segments at this depth.  In a large round 0 the
    // indices are the identity, so a separate gather streams the arena in
    // order; later rounds read it at random, and the count kernel of the first
    // partition level gathers the keys itself so that those reads overlap its
    // work (gather_fused).
    const bool fused_gather = gather_fused(this->fused_gather, fresh_round, h_ctr->gather_elems);
    if (n_large && !fused_gather) {
        LAUNCH(this, "seg_tiles",
               launch_seg_tiles(lcur, hcount(n_large), GATHER_TILE, ws.tile_base, st));
        LAUNCH(this, "gather", launch_gather(a, lcur, hcount(n_large), ws.tile_base, dc, g8, st));
    }
    uint32_t levels_this_round = 0;
    while (n_large) {
        // Every level strictly shrinks each range bucket (its splitter keys
        // leave for equality buckets), so this bound is never reached on
        // valid input; it turns a logic error into a status, not a hang.
        if (++levels_this_round > 4096)
            return fail(SSORT_EINTERNAL, "partition levels exceeded 4096");
        stats.partition_levels++;
        const bool first = fused_gather && levels_this_round == 1;
        const Count nl = hcount(n_large);
        LAUNCH(this, "sample",
               launch_sample(a, lcur, nl, ws.spl, ws.nspl, ws.tbl, ws.ntiles, ws.cm_size,
                             first, 0, st));
        LAUNCH(this, "scan_pair",
               launch_scan_pair(ws.ntiles, ws.tile_base, ws.cm_size, ws.cm_base, nl, st));
        LAUNCH(this, first ? "count_gather" : "count",
               launch_count(a, lcur, nl, ws.tile_base, ws.spl, ws.nspl, ws.tbl, ws.cm_base,
                            ws.cm, dc, first, g2, st));
        SS_TRY(scan(ws.cm, ws.cm, (uint32_t)(ws.cm_cap - 1), dcount(ws.cm_base + n_large)));
        LAUNCH(this, "scatter",
               launch_scatter(a, lcur, nl, ws.tile_base, ws.spl, ws.nspl, ws.tbl, ws.cm_base,
                              ws.cm, g2, st));
        LAUNCH(this, "emit",
               launch_emit(a, lcur, nl, ws.tile_base, ws.nspl, ws.cm_base, ws.cm, ws.W1, ws.W8,
                           SmallLists{{ws.S, ws.S2, ws.S3}}, lnext, ws.E, ws.B, nxt, dc, 0, st));
        SS_TRY(launch_small(a, nxt, done));  // segments known before this level
        SS_TRY(sync_counters());
        SS_TRY(fork_small());
        n_large = h_ctr->n_large_next;
        SS_CUDA(cudaMemsetAsync(&dc->n_large_next, 0, 4, st));
        std::swap(lcur, lnext);
    }
    SS_TRY(launch_small(a, nxt, done));  // the rest
    if (overlap_round) {
        SS_CUDA(cudaEventRecord(ev_join, side));
        SS_CUDA(cudaStreamWaitEvent(st, ev_join, 0));
        SS_CUDA(cudaEventRecord(ev_join2, side2));
        SS_CUDA(cudaStreamWaitEvent(st, ev_join2, 0));
    }
    LAUNCH(this, "boundary", launch_boundary(a, ws.B, dc, g4, st));
    SS_TRY(sync_counters());
    stats.small_segments +=
        h_ctr->n_w1 + h_ctr->n_w8 + h_ctr->n_small + h_ctr->n_small2 + h_ctr->n_small3;
    stats.partitioned += h_ctr->partitioned;
    stats.gather_elems += h_ctr->gather_elems;
    if (fused_gather) stats.gather_fused += h_ctr->gather_elems;
    stats.warp1_fresh += h_ctr->warp1_fresh;
    stats.warp1_deep += h_ctr->warp1_deep;
    stats.full_sorted += h_ctr->full_sorted;
    stats.window_saved += h_ctr->window_saved;
    stats.window_used += h_ctr->window_used;
    stats.warp1_keyed += h_ctr->warp1_keyed;
    stats.warp8_fresh += h_ctr->warp8_fresh;
    stats.warp8_keyed += h_ctr->warp8_keyed;
    stats.block_fresh += h_ctr->block_fresh;
    stats.block_keyed += h_ctr->block_keyed;
    stats.equal_moved += h_ctr->equal_moved;
    stats.equal_final += h_ctr->equal_final;
    stats.boundaries += h_ctr->n_bound;
    n_next = h_ctr->n_next;
    return SSORT_OK;
}

int ssort_ctx::run(const uint8_t *arena_p, uint64_t arena_bytes, const void *offs_p,
                   int off_width, uint32_t n, uint32_t *d_perm, uint32_t *d_lcp,
                   const uint32_t *d_inst, uint32_t ninst) {
    SS_TRY(reserve(n));
    // Saving key bytes 16..31 in round 0 pays where many strings share their
    // first 16 bytes and so enter round 1: decided without a device read, by
    // the arena's bytes per string and by the share of strings that entered
    // round 1 in this context's previous sort (none yet: length alone).
    // The copies are an optimisation: without device memory for them the sort
    // goes ahead without (the workspace itself was reserved first).
    key2 = nullptr;
    if (n >= KEY2_MIN_N && arena_bytes >= (uint64_t)KEY2_MIN_BYTES_PER_STRING * n &&
        (round1_live < 0 || round1_live >= KEY2_MIN_ROUND1_LIVE) &&
        ensure(key2_buf, (size_t)n * sizeof(ulonglong2)) == SSORT_OK)
        key2 = (ulonglong2 *)key2_buf.p;
    const int rc =
        run_ws(arena_p, arena_bytes, offs_p, off_width, n, d_perm, d_lcp, d_inst, ninst);
    key2 = nullptr;
    if (rc == SSORT_OK && n)
        round1_live = stats.rounds >= 2 ? (double)stats.live[1] / (double)n : 0.0;
    return rc;
}

// The round loop over an already laid-out workspace `ws`.  Every position's
// final index lands in d_perm (= idx[0]); every lcp entry is written exactly
// once: inside an on-chip sort or an equality bucket for pairs in the same
// leaf, by the boundary pass for pairs split by a partition, and lcp[0] = 0 up
// front.  The host waits for the device twice per round (segment counts after
// classification, and the next round's count) plus once per partition level.
// With an instance table (d_inst, ninst > 0) every instance starts as its own
// round-0 segment and the result indices are made instance-local at the end.
int ssort_ctx::run_ws(const uint8_t *arena_p, uint64_t arena_bytes, const void *offs_p,
                      int off_width, uint32_t n, uint32_t *d_perm, uint32_t *d_lcp,
                      const uint32_t *d_inst, uint32_t ninst) {
    SortArgs a{};
    a.arena = arena_p;
    a.arena_bytes = arena_bytes;
    a.offs = offs_p;
    a.off_width = off_width;
    a.n = n;
    a.idx[0] = d_perm;
    a.idx[1] = ws.idx1;
    a.key[0] = ws.key0;
    a.key[1] = ws.key1;
    a.lcp = d_lcp ? d_lcp : ws.lcp;
    a.bkt = ws.bkt;
    a.target_bucket = target_bucket;
    a.warp8_cap = warp8_cap;
    a.warp1_deep = warp1_deep;
    a.l2_prefetch = l2_prefetch ? 1u : 0u;
    a.scatter_staged_idx = scatter_variant;
    a.block_lean = block_lean;
    a.match_vote = match_vote ? 1u : 0u;
    a.warp_merge = warp_merge ? 1u : 0u;
    a.max_splitters = (1u << (digit_bits - 1)) - 1;
    std::copy(std::begin(class_targets), std::end(class_targets), std::begin(a.target_by_class));
    a.key2 = key2;

    // The device-driven loop: not while profiling (per-kernel events need
    // host launches) and not for the server's per-round calls.
    if (graph_mode && !prof && graph_wanted(a, d_inst != nullptr))
        return run_graph(a, n, d_inst, ninst);

    Seg *cur = ws.R, *nxt = ws.N;
    Counters *dc = ws.ctr;

    LAUNCH(this, "iota", launch_iota(d_perm, n, st));
    SS_CUDA(cudaMemsetAsync(a.lcp, 0, 4, st));
    uint32_t n_cur = 1;
    if (d_inst) {
        SS_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), st));
        LAUNCH(this, "init_batch", launch_init_batch(d_inst, ninst, cur, a.lcp, dc, st));
        SS_TRY(sync_counters());
        n_cur = h_ctr->n_next;
    } else {
        if (n < 2) return SSORT_OK;
        Seg first{0, n, 0, 0};
        SS_CUDA(cudaMemcpyAsync(cur, &first, sizeof(Seg), cudaMemcpyHostToDevice, st));
    }
    uint32_t round_no = 0;
    while (n_cur) {
        uint32_t n_next = 0;
        SS_TRY(round(a, cur, n_cur, nxt, n_next, round_no));
        n_cur = n_next;
        std::swap(cur, nxt);
        ++round_no;
    }
    stats.rounds = round_no;
    if (d_inst) LAUNCH(this, "localize", launch_localize(d_perm, n, d_inst, ninst, st));
    return SSORT_OK;
}

// Copies `bytes` of ordinary (pageable) host memory to the device on st
// through two pinned chunks: the host threads copy chunk k + 1 into one while
// the DMA engine moves chunk k from the other, so the transfer runs at the
// rate of the slower of the two instead of the driver's pageable staging.
// Returns with the last transfer queued (not complete); the chunks are
// reused by the next call only after their events.
int ssort_ctx::copy_pageable(void *d_dst, const void *h_src, uint64_t bytes) {
    constexpr uint64_t CHUNK = 64ull << 20;
    if (bytes < 2 * CHUNK) {  // small: the driver's own path is as good
        SS_CUDA(cudaMemcpyAsync(d_dst, h_src, bytes, cudaMemcpyHostToDevice, st));
        return SSORT_OK;
    }
    for (int b = 0; b < 2; ++b) {
        SS_TRY(ensure_host(h_stage[b], CHUNK));
        if (!ev_stage[b]) SS_CUDA(cudaEventCreateWithFlags(&ev_stage[b], cudaEventDisableTiming));
    }
    const unsigned char *src = (const unsigned char *)h_src;
    unsigned char *dst = (unsigned char *)d_dst;
    uint64_t k = 0;
    for (uint64_t at = 0; at < bytes; at += CHUNK, ++k) {
        const int b = (int)(k & 1);
        const uint64_t len = std::min(CHUNK, bytes - at);
        // the chunk's previous transfer (two chunks back) has finished
        SS_CUDA(cudaEventSynchronize(ev_stage[b]));
        unsigned char *stage = (unsigned char *)h_stage[b].p;
        const int64_t pieces = 64;
        const uint64_t piece = (len + pieces - 1) / pieces;
#pragma omp parallel for
        for (int64_t q = 0; q < pieces; ++q) {
            const uint64_t o = (uint64_t)q * piece;
            if (o < len) std::memcpy(stage + o, src + at + o, std::min(piece, len - o));
        }
        SS_CUDA(cudaMemcpyAsync(dst + at, stage, len, cudaMemcpyHostToDevice, st));
        SS_CUDA(cudaEventRecord(ev_stage[b], st));
    }
    return SSORT_OK;
}

// ---------------------------------------------------------------------------
namespace {

int validate_common(ssort_ctx *ctx, int off_width, uint64_t n) {
    if (!ctx) return fail(SSORT_EINVAL, "null context");
    if (off_width != 4 && off_width != 8) return fail(SSORT_EINVAL, "off_width must be 4 or 8");
    if (n > SSORT_MAX_N) return fail(SSORT_EINVAL, "n exceeds SSORT_MAX_N");
    return SSORT_OK;
}

uint32_t size_class(uint64_t n) { return n ? 63u - (uint32_t)__builtin_clzll(n) : 0u; }
uint32_t entropy_class(double bits) { return bits < 2.0 ? 0u : (bits < 4.0 ? 1u : 2u); }

// Applies autotuned values recorded for this input's size and entropy class.
// A batched sort (many instances of many sizes) also gets, per segment size
// class, the range-bucket size tuned for that class and the batch's entropy
// class, so that each instance is partitioned as a plain sort of its size
// would be.
int apply_tuning(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                 const void *d_offs, int off_width, uint64_t n, bool batched) {
    std::fill(std::begin(ctx->class_targets), std::end(ctx->class_targets), uint16_t(0));
    if (ctx->tuned.empty() || ctx->tuning || n < 2) return SSORT_OK;
    if (batched) {
        double bits = 0;
        SS_TRY(ctx->sample_entropy(d_arena, arena_bytes, d_offs, off_width, (uint32_t)n, bits));
        const uint32_t ec = entropy_class(bits);
        for (uint32_t c = 0; c < 32; ++c) {
            auto t = ctx->tuned.find(c * 4 + ec);
            if (t != ctx->tuned.end()) ctx->class_targets[c] = (uint16_t)t->second.target_bucket;
        }
    }
    const uint32_t sc = size_class(n);
    uint32_t classes = 0, only = 0;
    for (uint32_t e = 0; e < 3; ++e)
        if (ctx->tuned.count(sc * 4 + e)) {
            ++classes;
            only = e;
        }
    if (!classes) return SSORT_OK;
    // One recorded entropy class for this size: use it without sampling.
    uint32_t ec = only;
    if (classes > 1) {
        double bits = 0;
        SS_TRY(ctx->sample_entropy(d_arena, arena_bytes, d_offs, off_width, (uint32_t)n, bits));
        ec = entropy_class(bits);
    }
    auto it = ctx->tuned.find(sc * 4 + ec);
    if (it == ctx->tuned.end()) return SSORT_OK;
    ctx->target_bucket = it->second.target_bucket;
    ctx->warp8_cap = it->second.warp8_cap;
    ctx->overlap = it->second.overlap;
    ctx->fused_gather = it->second.fused_gather;
    ctx->digit_bits = it->second.digit_bits;
    ctx->block_prefetch = it->second.block_prefetch;
    ctx->l2_prefetch = it->second.l2_prefetch;
    ctx->graph_mode = it->second.graph;
    ctx->block_lean = it->second.block_lean;
    return SSORT_OK;
}

int sort_device_impl(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                     const void *d_offs, int off_width, uint64_t n, uint32_t *d_perm,
                     uint32_t *d_lcp, const uint32_t *d_inst = nullptr, uint32_t ninst = 0) {
    SS_TRY(apply_tuning(ctx, d_arena, arena_bytes, d_offs, off_width, n, d_inst != nullptr));
    ctx->stats = ssort_stats{};
    ctx->stats.n = n;
    SS_CUDA(cudaEventRecord(ctx->ev_start, ctx->st));
    int rc = ctx->run(d_arena, arena_bytes, d_offs, off_width, (uint32_t)n, d_perm, d_lcp, d_inst,
                      ninst);
    if (rc != SSORT_OK) {
        cudaStreamSynchronize(ctx->st);
        if (ctx->side) cudaStreamSynchronize(ctx->side);
        if (ctx->side2) cudaStreamSynchronize(ctx->side2);
        if (ctx->hp) cudaStreamSynchronize(ctx->hp);
        ctx->recs.clear();
        ctx->ev_used = 0;
        return rc;
    }
    SS_CUDA(cudaEventRecord(ctx->ev_stop, ctx->st));
    SS_CUDA(cudaStreamSynchronize(ctx->st));
    float ms = 0;
    cudaEventElapsedTime(&ms, ctx->ev_start, ctx->ev_stop);
    ctx->stats.device_ms = ms;
    if (ctx->prof) ctx->prof_collect();
    size_t held = 0;
    for (DBuf *b : {&ctx->ws_buf, &ctx->arena, &ctx->offs, &ctx->perm, &ctx->inst, &ctx->aux,
                     &ctx->aux2})
        held += b->cap;
    ctx->stats.device_bytes = held;
    return SSORT_OK;
}

// Readable mappings of this process, for the drop-in's one-span fast path.
bool span_is_readable(uintptr_t lo, uintptr_t hi) {
    FILE *f = std::fopen("/proc/self/maps", "r");
    if (!f) return false;
    std::vector<std::pair<uintptr_t, uintptr_t>> rd;
    char line[512];
    while (std::fgets(line, sizeof line, f)) {
        unsigned long a, b;
        char perm[8] = {0};
        if (std::sscanf(line, "%lx-%lx %7s", &a, &b, perm) == 3 && perm[0] == 'r')
            rd.emplace_back((uintptr_t)a, (uintptr_t)b);
    }
    std::fclose(f);
    std::sort(rd.begin(), rd.end());
    uintptr_t cur = lo;
    for (auto &m : rd) {
        if (m.second <= cur) continue;
        if (m.first > cur) return false;
        cur = m.second;
        if (cur >= hi) return true;
    }
    return cur >= hi;
}

}  // namespace

extern "C" {

const char *ssort_strerror(int status) {
    switch (status) {
        case SSORT_OK: return "ok";
        case SSORT_EINVAL: return "invalid argument";
        case SSORT_ENOMEM: return "out of memory";
        case SSORT_ECUDA: return "CUDA error";
        case SSORT_ENODEV: return "no CUDA device";
        case SSORT_EINTERNAL: return "internal error";
        default: return "unknown status";
    }
}

const char *ssort_last_error(void) { return g_last_error.c_str(); }

int ssort_ctx_create(int device, ssort_ctx **out) {
    if (!out) return fail(SSORT_EINVAL, "null output pointer");
    *out = nullptr;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(SSORT_ENODEV, "no CUDA device available");
    }
    if (device < 0 || device >= ndev) return fail(SSORT_EINVAL, "device index out of range");
    ssort_ctx *ctx = new ssort_ctx();
    ctx->device = device;
    int rc = with_device(ctx, [&]() -> int {
        SS_CUDA(cudaDeviceGetAttribute(&ctx->num_sms, cudaDevAttrMultiProcessorCount, device));
        SS_CUDA(cudaStreamCreateWithFlags(&ctx->own_stream, cudaStreamNonBlocking));
        // The partition levels (hp) and the on-chip sorts (side) of a round run
        // on two streams of equal priority: giving the partition the higher
        // one measured 0.6 % slower on 50 M URLs.
        SS_CUDA(cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
        SS_CUDA(cudaStreamCreateWithFlags(&ctx->side2, cudaStreamNonBlocking));
        SS_CUDA(cudaEventCreateWithFlags(&ctx->ev_join2, cudaEventDisableTiming));
        SS_CUDA(cudaStreamCreateWithFlags(&ctx->hp, cudaStreamNonBlocking));
        SS_CUDA(cudaEventCreateWithFlags(&ctx->ev_fork, cudaEventDisableTiming));
        SS_CUDA(cudaEventCreateWithFlags(&ctx->ev_join, cudaEventDisableTiming));
        SS_CUDA(cudaEventCreateWithFlags(&ctx->ev_round, cudaEventDisableTiming));
        SS_CUDA(cudaEventCreate(&ctx->ev_start));
        SS_CUDA(cudaEventCreate(&ctx->ev_stop));
        ctx->st = ctx->own_stream;
        return SSORT_OK;
    });
    if (rc != SSORT_OK) {
        delete ctx;
        return rc;
    }
    *out = ctx;
    return SSORT_OK;
}

void ssort_ctx_destroy(ssort_ctx *ctx) {
    if (!ctx) return;
    with_device(ctx, [&]() -> int {
        if (ctx->own_stream) cudaStreamSynchronize(ctx->own_stream);
        ctx->graph_release();
        for (cudaStream_t c : ctx->cap)
            if (c) cudaStreamDestroy(c);
        if (ctx->h_gs) cudaFreeHost(ctx->h_gs);
        for (DBuf *b : {&ctx->ws_buf, &ctx->arena, &ctx->offs, &ctx->perm, &ctx->inst, &ctx->aux,
                     &ctx->aux2})
            if (b->p) cudaFree(b->p);
        for (HBuf *b : {&ctx->h_offs, &ctx->h_arena, &ctx->h_perm, &ctx->h_stage[0],
                        &ctx->h_stage[1]})
            if (b->p) cudaFreeHost(b->p);
        for (cudaEvent_t e : ctx->ev_stage)
            if (e) cudaEventDestroy(e);
        if (ctx->h_ctr) cudaFreeHost(ctx->h_ctr);
        if (ctx->h_hist) cudaFreeHost(ctx->h_hist);
        if (ctx->hist_buf.p) cudaFree(ctx->hist_buf.p);
        for (auto e : ctx->ev_pool) cudaEventDestroy(e);
        if (ctx->ev_start) cudaEventDestroy(ctx->ev_start);
        if (ctx->ev_stop) cudaEventDestroy(ctx->ev_stop);
        if (ctx->side) cudaStreamSynchronize(ctx->side);
        if (ctx->side2) cudaStreamSynchronize(ctx->side2);
        if (ctx->hp) cudaStreamSynchronize(ctx->hp);
        if (ctx->ev_fork) cudaEventDestroy(ctx->ev_fork);
        if (ctx->ev_join) cudaEventDestroy(ctx->ev_join);
        if (ctx->ev_join2) cudaEventDestroy(ctx->ev_join2);
        if (ctx->ev_round) cudaEventDestroy(ctx->ev_round);
        if (ctx->side) cudaStreamDestroy(ctx->side);
        if (ctx->side2) cudaStreamDestroy(ctx->side2);
        if (ctx->hp) cudaStreamDestroy(ctx->hp);
        if (ctx->own_stream) cudaStreamDestroy(ctx->own_stream);
        return SSORT_OK;
    });
    delete ctx;
}

int ssort_sort_device(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                      const void *d_offs, int off_width, uint64_t n, uint32_t *d_perm,
                      uint32_t *d_lcp, void *stream) {
    SS_TRY(validate_common(ctx, off_width, n));
    if (n == 0) return SSORT_OK;
    if (!d_arena || !d_offs || !d_perm) return fail(SSORT_EINVAL, "null device buffer");
    if (((uintptr_t)d_arena & 15) != 0)
        return fail(SSORT_EINVAL, "arena must be 16-byte aligned");
    return with_device(ctx, [&]() -> int {
        ctx->st = stream ? (cudaStream_t)stream : ctx->own_stream;
        int rc = sort_device_impl(ctx, d_arena, arena_bytes, d_offs, off_width, n, d_perm, d_lcp);
        ctx->st = ctx->own_stream;
        return rc;
    });
}

int ssort_sort_batch_device(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                            const void *d_offs, int off_width, uint64_t n,
                            const uint32_t *d_inst_start, uint32_t ninst, uint32_t *d_perm,
                            uint32_t *d_lcp, void *stream) {
    SS_TRY(validate_common(ctx, off_width, n));
    if (n == 0) return SSORT_OK;
    if (!d_arena || !d_offs || !d_perm || !d_inst_start)
        return fail(SSORT_EINVAL, "null device buffer");
    if (ninst == 0) return fail(SSORT_EINVAL, "no instances");
    if (((uintptr_t)d_arena & 15) != 0)
        return fail(SSORT_EINVAL, "arena must be 16-byte aligned");
    return with_device(ctx, [&]() -> int {
        ctx->st = stream ? (cudaStream_t)stream : ctx->own_stream;
        int rc = sort_device_impl(ctx, d_arena, arena_bytes, d_offs, off_width, n, d_perm, d_lcp,
                                  d_inst_start, ninst);
        ctx->st = ctx->own_stream;
        return rc;
    });
}

int ssort_sort_batch_host(ssort_ctx *ctx, const uint8_t *arena, uint64_t arena_bytes,
                          const void *offs, int off_width, uint64_t n, const uint32_t *inst_start,
                          uint32_t ninst, uint32_t *perm, uint32_t *lcp) {
    SS_TRY(validate_common(ctx, off_width, n));
    if (n == 0) return SSORT_OK;
    if (!arena || !offs || !perm || !inst_start) return fail(SSORT_EINVAL, "null host buffer");
    if (ninst == 0) return fail(SSORT_EINVAL, "no instances");
    if (inst_start[0] != 0 || inst_start[ninst] != n)
        return fail(SSORT_EINVAL, "instance table must start at 0 and end at n");
    for (uint32_t i = 0; i < ninst; ++i)
        if (inst_start[i + 1] < inst_start[i])
            return fail(SSORT_EINVAL, "instance table must be non-decreasing");
    return with_device(ctx, [&]() -> int {
        ctx->st = ctx->own_stream;
        SS_TRY(ctx->ensure(ctx->arena, arena_bytes + 16));
        SS_TRY(ctx->ensure(ctx->offs, n * off_width));
        SS_TRY(ctx->ensure(ctx->perm, n * 4 * (lcp ? 2 : 1)));
        SS_TRY(ctx->ensure(ctx->inst, ((size_t)ninst + 1) * 4));
        uint8_t *d_arena = (uint8_t *)ctx->arena.p;
        uint32_t *d_perm = (uint32_t *)ctx->perm.p;
        uint32_t *d_lcp = lcp ? d_perm + n : nullptr;
        SS_CUDA(cudaMemcpyAsync(d_arena, arena, arena_bytes, cudaMemcpyHostToDevice, ctx->st));
        SS_CUDA(cudaMemsetAsync(d_arena + arena_bytes, 0, 16, ctx->st));
        SS_CUDA(cudaMemcpyAsync(ctx->offs.p, offs, n * off_width, cudaMemcpyHostToDevice, ctx->st));
        SS_CUDA(cudaMemcpyAsync(ctx->inst.p, inst_start, ((size_t)ninst + 1) * 4,
                                cudaMemcpyHostToDevice, ctx->st));
        SS_TRY(sort_device_impl(ctx, d_arena, arena_bytes + 16, ctx->offs.p, off_width, n, d_perm,
                                d_lcp, (const uint32_t *)ctx->inst.p, ninst));
        SS_CUDA(cudaMemcpyAsync(perm, d_perm, n * 4, cudaMemcpyDeviceToHost, ctx->st));
        if (lcp) SS_CUDA(cudaMemcpyAsync(lcp, d_lcp, n * 4, cudaMemcpyDeviceToHost, ctx->st));
        SS_CUDA(cudaStreamSynchronize(ctx->st));
        return SSORT_OK;
    });
}

int ssort_sort_host(ssort_ctx *ctx, const uint8_t *arena, uint64_t arena_bytes, const void *offs,
                    int off_width, uint64_t n, uint32_t *perm, uint32_t *lcp) {
    SS_TRY(validate_common(ctx, off_width, n));
    if (n == 0) return SSORT_OK;
    if (!arena || !offs || !perm) return fail(SSORT_EINVAL, "null host buffer");
    return with_device(ctx, [&]() -> int {
        ctx->st = ctx->own_stream;
        // Device arena: the bytes plus 16 zero bytes of padding.
        SS_TRY(ctx->ensure(ctx->arena, arena_bytes + 16));
        SS_TRY(ctx->ensure(ctx->perm, n * 4 * (lcp ? 2 : 1)));
        uint8_t *d_arena = (uint8_t *)ctx->arena.p;
        uint32_t *d_perm = (uint32_t *)ctx->perm.p;
        uint32_t *d_lcp = lcp ? d_perm + n : nullptr;
        SS_CUDA(cudaMemcpyAsync(d_arena, arena, arena_bytes, cudaMemcpyHostToDevice, ctx->st));
        SS_CUDA(cudaMemsetAsync(d_arena + arena_bytes, 0, 16, ctx->st));
        // 8-byte offsets into an arena below 4 GB cross the link as 4-byte
        // ones: the host threads narrow them into a pinned buffer while the
        // copy engine moves the arena, halving the offsets' share of the
        // transfer.  If any offset does not fit, the 8-byte ones are sent.
        int ow = off_width;
        const void *src = offs;
        if (off_width == 8 && arena_bytes + 16 <= 0xFFFFFFFFull && n >= NARROW_OFFS_MIN_N) {
            SS_TRY(ctx->ensure_host(ctx->h_offs, n * 4));
            uint32_t *o32 = (uint32_t *)ctx->h_offs.p;
            const uint64_t *o64 = (const uint64_t *)offs;
            const int64_t nn = (int64_t)n;
            uint64_t mx = 0;
#pragma omp parallel for reduction(max : mx)
            for (int64_t i = 0; i < nn; ++i) {
                const uint64_t v = o64[i];
                mx = std::max(mx, v);
                o32[i] = (uint32_t)v;
            }
            if (mx <= 0xFFFFFFFFull) {
                ow = 4;
                src = o32;
            }
        }
        SS_TRY(ctx->ensure(ctx->offs, n * ow));
        SS_CUDA(cudaMemcpyAsync(ctx->offs.p, src, n * ow, cudaMemcpyHostToDevice, ctx->st));
        SS_TRY(sort_device_impl(ctx, d_arena, arena_bytes + 16, ctx->offs.p, ow, n, d_perm,
                                d_lcp));
        SS_CUDA(cudaMemcpyAsync(perm, d_perm, n * 4, cudaMemcpyDeviceToHost, ctx->st));
        if (lcp) SS_CUDA(cudaMemcpyAsync(lcp, d_lcp, n * 4, cudaMemcpyDeviceToHost, ctx->st));
        SS_CUDA(cudaStreamSynchronize(ctx->st));
        return SSORT_OK;
    });
}

int ssort_sort_strings(ssort_ctx *ctx, unsigned char **strings, size_t n, uint32_t *lcp_out) {
    if (!ctx) return fail(SSORT_EINVAL, "null context");
    if (n > SSORT_MAX_N) return fail(SSORT_EINVAL, "n exceeds SSORT_MAX_N");
    if (n == 0) return SSORT_OK;
    if (!strings) return fail(SSORT_EINVAL, "null string array");
    for (size_t i = 0; i < n; ++i)
        if (!strings[i]) return fail(SSORT_EINVAL, "null string pointer at index " + std::to_string(i));
    if (n == 1) {
        if (lcp_out) lcp_out[0] = 0;
        return SSORT_OK;
    }
    return with_device(ctx, [&]() -> int {
        ctx->st = ctx->own_stream;
        const int64_t nn = (int64_t)n;
        // One readable span holding every string (sortstring's single text
        // buffer, src/sortstring.c:310-335): ship the span as is.  Otherwise
        // (e.g. separately strdup'd strings, unit-test/main.cpp:220-270) pack
        // the strings into a pinned staging arena.
        uintptr_t lo = UINTPTR_MAX, hi_start = 0;
#pragma omp parallel for reduction(min : lo) reduction(max : hi_start) if (nn > 100000)
        for (int64_t i = 0; i < nn; ++i) {
            const uintptr_t p = (uintptr_t)strings[i];
            lo = std::min(lo, p);
            hi_start = std::max(hi_start, p);
        }
        const uintptr_t hi = hi_start + std::strlen((const char *)hi_start) + 1;
        const uint64_t span = hi - lo;
        size_t free_b = 0, total_b = 0;
        cudaMemGetInfo(&free_b, &total_b);
        const bool use_span = span <= (uint64_t)free_b / 4 && span_is_readable(lo, hi);
        const uint8_t *src;
        uint64_t bytes;
        int ow;
        if (use_span) {
            ow = span < 0xFFFFFFF0ull ? 4 : 8;
            SS_TRY(ctx->ensure_host(ctx->h_offs, n * ow));
            if (ow == 4) {
                uint32_t *o = (uint32_t *)ctx->h_offs.p;
#pragma omp parallel for if (nn > 100000)
                for (int64_t i = 0; i < nn; ++i) o[i] = (uint32_t)((uintptr_t)strings[i] - lo);
            } else {
                uint64_t *o = (uint64_t *)ctx->h_offs.p;
#pragma omp parallel for if (nn > 100000)
                for (int64_t i = 0; i < nn; ++i) o[i] = (uint64_t)((uintptr_t)strings[i] - lo);
            }
            src = (const uint8_t *)lo;
            bytes = span;
        } else {
            std::vector<uint64_t> len(n);
#pragma omp parallel for if (nn > 100000)
            for (int64_t i = 0; i < nn; ++i) len[i] = std::strlen((const char *)strings[i]) + 1;
            uint64_t total = 0;
            for (size_t i = 0; i < n; ++i) {
                const uint64_t l = len[i];
                len[i] = total;
                total += l;
            }
            ow = total < 0xFFFFFFF0ull ? 4 : 8;
            SS_TRY(ctx->ensure_host(ctx->h_offs, n * ow));
            SS_TRY(ctx->ensure_host(ctx->h_arena, total));
            uint8_t *dst = (uint8_t *)ctx->h_arena.p;
#pragma omp parallel for if (nn > 100000)
            for (int64_t i = 0; i < nn; ++i) {
                const uint64_t o = len[i];
                const uint64_t l = (i + 1 < nn ? len[i + 1] : total) - o;
                std::memcpy(dst + o, strings[i], l);
                if (ow == 4)
                    ((uint32_t *)ctx->h_offs.p)[i] = (uint32_t)o;
                else
                    ((uint64_t *)ctx->h_offs.p)[i] = o;
            }
            src = dst;
            bytes = total;
        }
        SS_TRY(ctx->ensure_host(ctx->h_perm, n * 4));
        uint32_t *perm = (uint32_t *)ctx->h_perm.p;
        // Device copies of the arena, offsets and results.
        SS_TRY(ctx->ensure(ctx->arena, bytes + 16));
        SS_TRY(ctx->ensure(ctx->offs, n * ow));
        SS_TRY(ctx->ensure(ctx->perm, n * 4 * (lcp_out ? 2 : 1)));
        uint8_t *d_arena = (uint8_t *)ctx->arena.p;
        uint32_t *d_perm = (uint32_t *)ctx->perm.p;
        uint32_t *d_lcp = lcp_out ? d_perm + n : nullptr;
        // The caller's span is ordinary memory: staged through pinned chunks.
        if (use_span)
            SS_TRY(ctx->copy_pageable(d_arena, src, bytes));
        else
            SS_CUDA(cudaMemcpyAsync(d_arena, src, bytes, cudaMemcpyHostToDevice, ctx->st));
        SS_CUDA(cudaMemsetAsync(d_arena + bytes, 0, 16, ctx->st));
        SS_CUDA(cudaMemcpyAsync(ctx->offs.p, ctx->h_offs.p, n * ow, cudaMemcpyHostToDevice,
                                ctx->st));
        SS_TRY(sort_device_impl(ctx, d_arena, bytes + 16, ctx->offs.p, ow, n, d_perm, d_lcp));
        if (lcp_out)
            SS_CUDA(cudaMemcpyAsync(lcp_out, d_lcp, n * 4, cudaMemcpyDeviceToHost, ctx->st));
        if (use_span) {
            // One span: the sorted strings' offsets into it (in the
            // offsets' own width) come back in order, and the pointer array
            // is rewritten sequentially (no random gather through a copy of
            // the old array).
            SS_TRY(ctx->ensure(ctx->aux2, n * ow));
            SS_TRY(ctx->ensure_host(ctx->h_arena, n * ow));  // unused by the span path
            LAUNCH(ctx, "sorted_offs",
                   launch_sorted_offs(d_perm, ctx->offs.p, ow, n, ctx->aux2.p, ow, ctx->st));
            SS_CUDA(cudaMemcpyAsync(ctx->h_arena.p, ctx->aux2.p, n * ow, cudaMemcpyDeviceToHost,
                                    ctx->st));
            SS_CUDA(cudaStreamSynchronize(ctx->st));
            unsigned char *base = (unsigned char *)lo;
            if (ow == 4) {
                const uint32_t *so = (const uint32_t *)ctx->h_arena.p;
#pragma omp parallel for if (nn > 100000)
                for (int64_t i = 0; i < nn; ++i) strings[i] = base + so[i];
            } else {
                const uint64_t *so = (const uint64_t *)ctx->h_arena.p;
#pragma omp parallel for if (nn > 100000)
                for (int64_t i = 0; i < nn; ++i) strings[i] = base + so[i];
            }
            return SSORT_OK;
        }
        SS_CUDA(cudaMemcpyAsync(perm, d_perm, n * 4, cudaMemcpyDeviceToHost, ctx->st));
        SS_CUDA(cudaStreamSynchronize(ctx->st));
        std::vector<unsigned char *> orig(strings, strings + n);
#pragma omp parallel for if (nn > 100000)
        for (int64_t i = 0; i < nn; ++i) strings[i] = orig[perm[i]];
        return SSORT_OK;
    });
}

int ssort_get_stats(const ssort_ctx *ctx, ssort_stats *out) {
    if (!ctx || !out) return fail(SSORT_EINVAL, "null argument");
    *out = ctx->stats;
    return SSORT_OK;
}

int ssort_set_param(ssort_ctx *ctx, int param, int64_t value) {
    if (!ctx) return fail(SSORT_EINVAL, "null context");
    switch (param) {
        case SSORT_PARAM_TARGET_BUCKET:
            if (value < 32 || value > SMALL_CAP) return fail(SSORT_EINVAL, "target_bucket out of range");
            ctx->target_bucket = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_WARP8_CAP:
            if (value < 64 || value > WARP8_CAP)
                return fail(SSORT_EINVAL, "warp8_cap out of range (64..256)");
            ctx->warp8_cap = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_OVERLAP:
            if (value != 0 && value != 1) return fail(SSORT_EINVAL, "overlap must be 0 or 1");
            ctx->overlap = value != 0;
            return SSORT_OK;
        case SSORT_PARAM_FUSED_GATHER:
            if (value < 0 || value > 2) return fail(SSORT_EINVAL, "fused_gather must be 0, 1 or 2");
            ctx->fused_gather = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_DIGIT_BITS:
            if (value < 8 || value > 10) return fail(SSORT_EINVAL, "digit_bits out of range (8..10)");
            ctx->digit_bits = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_SCAN:
            if (value != 0 && value != 1) return fail(SSORT_EINVAL, "scan must be 0 or 1");
            ctx->scan_lookback = value != 0;
            return SSORT_OK;
        case SSORT_PARAM_WARP_MERGE:
            if (value != 0 && value != 1) return fail(SSORT_EINVAL, "warp_merge must be 0 or 1");
            ctx->warp_merge = value != 0;
            return SSORT_OK;
        case SSORT_PARAM_MATCH_VOTE:
            if (value != 0 && value != 1) return fail(SSORT_EINVAL, "match_vote must be 0 or 1");
            ctx->match_vote = value != 0;
            return SSORT_OK;
        case SSORT_PARAM_BLOCK_LEAN:
            if (value < 0 || value > 2) return fail(SSORT_EINVAL, "block_lean must be 0, 1 or 2");
            ctx->block_lean = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_SCATTER:
            if (value < 0 || value > 2) return fail(SSORT_EINVAL, "scatter must be 0, 1 or 2");
            ctx->scatter_variant = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_L2_PREFETCH:
            if (value != 0 && value != 1) return fail(SSORT_EINVAL, "l2_prefetch must be 0 or 1");
            ctx->l2_prefetch = value != 0;
            return SSORT_OK;
        case SSORT_PARAM_GRAPH:
            if (value < 0 || value > 2) return fail(SSORT_EINVAL, "graph must be 0, 1 or 2");
            ctx->graph_mode = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_GRAPH_MAX_LEVELS:
            if (value < 1 || value > (int64_t)GRAPH_MAX_LEVELS)
                return fail(SSORT_EINVAL, "graph_max_levels out of range (1..4096)");
            ctx->graph_max_levels = (uint32_t)value;
            return SSORT_OK;
        case SSORT_PARAM_BLOCK_PREFETCH:
            if (value != 0 && value != 1) return fail(SSORT_EINVAL, "block_prefetch must be 0 or 1");
            ctx->block_prefetch = value != 0;
            return SSORT_OK;
        case SSORT_PARAM_WARP1_DEEP:
            if (value < 0 || value > WARP1_DEEP_MAX)
                return fail(SSORT_EINVAL, "warp1_deep out of range (0..4096)");
            ctx->warp1_deep = (uint32_t)value;
            return SSORT_OK;
        default:
            return fail(SSORT_EINVAL, "unknown parameter");
    }
}

int ssort_set_profiling(ssort_ctx *ctx, int enabled) {
    if (!ctx) return fail(SSORT_EINVAL, "null context");
    ctx->prof = enabled != 0;
    if (!ctx->prof) ctx->ktimes.clear();
    return SSORT_OK;
}

int ssort_get_kernel_times(const ssort_ctx *ctx, const char **names, double *total_ms,
                           uint64_t *launches, int max) {
    if (!ctx) return fail(SSORT_EINVAL, "null context");
    int i = 0;
    for (auto &kv : ctx->ktimes) {
        if (i < max) {
            if (names) names[i] = kv.first.c_str();
            if (total_ms) total_ms[i] = kv.second.first;
            if (launches) launches[i] = kv.second.second;
        }
        ++i;
    }
    return i;
}

// The drop-in routine (struct routine::f, src/routine.h:33).
void msd_gpu(unsigned char **strings, size_t n) {
    static std::mutex mu;
    static ssort_ctx *ctx = nullptr;
    if (n < 2) return;
    std::lock_guard<std::mutex> lock(mu);
    if (!ctx) {
        int dev = 0;
        cudaGetDevice(&dev);
        int rc = ssort_ctx_create(dev, &ctx);
        if (rc != SSORT_OK) {
            std::fprintf(stderr, "msd_gpu: %s: %s\n", ssort_strerror(rc), ssort_last_error());
            std::abort();
        }
    }
    int rc = ssort_sort_strings(ctx, strings, n, nullptr);
    if (rc != SSORT_OK) {
        std::fprintf(stderr, "msd_gpu: %s: %s\n", ssort_strerror(rc), ssort_last_error());
        std::abort();
    }
}

}  // extern "C"

// ---- text inputs ---------------------------------------------------------------
namespace {

// Count phase of the delimited modes: per-tile delimiter counts (kept in
// ctx->aux for the write phase) and their total.
int text_count(ssort_ctx *ctx, const uint8_t *d_text, uint64_t len, uint8_t delim,
               uint64_t *n_out) {
    const uint64_t tiles = text_tiles(len);
    *n_out = 0;
    if (!tiles) return SSORT_OK;
    if (tiles >= 0xFFFFFFF0ull) return fail(SSORT_EINVAL, "text too long");
    const uint32_t nt = (uint32_t)tiles;
    const size_t parts = scan_partials_needed(nt);
    SS_TRY(ctx->ensure(ctx->aux, 256 + ((size_t)nt + 1) * 4 + 256 + parts * 4));
    unsigned long long *d_total = (unsigned long long *)ctx->aux.p;
    uint32_t *d_tiles = (uint32_t *)((unsigned char *)ctx->aux.p + 256);
    SS_CUDA(cudaMemsetAsync(d_total, 0, 8, ctx->st));
    LAUNCH(ctx, "text_count", launch_text_count(d_text, len, delim, d_tiles, d_total, ctx->st));
    unsigned long long total = 0;
    SS_CUDA(cudaMemcpyAsync(&total, d_total, 8, cudaMemcpyDeviceToHost, ctx->st));
    SS_CUDA(cudaStreamSynchronize(ctx->st));
    *n_out = total;
    return SSORT_OK;
}

// Write phase: string starts from the scanned tile counts of text_count.
int text_write(ssort_ctx *ctx, uint8_t *d_text, uint64_t len, uint8_t delim, uint64_t n,
               void *d_offs, int off_width) {
    const uint32_t nt = (uint32_t)text_tiles(len);
    uint32_t *d_tiles = (uint32_t *)((unsigned char *)ctx->aux.p + 256);
    uint32_t *d_parts =
        (uint32_t *)((unsigned char *)ctx->aux.p + 256 + (((size_t)nt + 1) * 4 + 255) / 256 * 256);
    LAUNCH(ctx, "scan", launch_scan(d_tiles, d_tiles, nt, hcount(nt), d_parts, ctx->st));
    LAUNCH(ctx, "text_starts",
           launch_text_starts(d_text, len, delim, d_tiles, n, d_offs, off_width, ctx->st));
    return SSORT_OK;
}

int text_check(ssort_ctx *ctx, uint64_t text_len, int mode, int off_width, uint64_t *n_out) {
    if (!ctx) return fail(SSORT_EINVAL, "null context");
    if (!n_out) return fail(SSORT_EINVAL, "null count pointer");
    if (mode != SSORT_TEXT_LINES && mode != SSORT_TEXT_RAW && mode != SSORT_TEXT_SUFFIXES)
        return fail(SSORT_EINVAL, "unknown text mode");
    if (off_width != 4 && off_width != 8) return fail(SSORT_EINVAL, "off_width must be 4 or 8");
    if (off_width == 4 && text_len >= (1ull << 32))
        return fail(SSORT_EINVAL, "4-byte offsets need a text shorter than 2^32 bytes");
    return SSORT_OK;
}

int text_fits(uint64_t n, uint64_t cap) {
    if (n > SSORT_MAX_N) return fail(SSORT_EINVAL, "text holds more strings than SSORT_MAX_N");
    if (n > cap)
        return fail(SSORT_EINVAL, "offset capacity too small: the text holds " +
                                      std::to_string(n) + " strings");
    return SSORT_OK;
}

}  // namespace

extern "C" {

int ssort_text_offsets_device(ssort_ctx *ctx, uint8_t *d_text, uint64_t text_len, int mode,
                              void *d_offs, int off_width, uint64_t cap, uint64_t *n_out,
                              void *stream) {
    SS_TRY(text_check(ctx, text_len, mode, off_width, n_out));
    *n_out = 0;
    if (!text_len) return SSORT_OK;
    if (!d_text || !d_offs) return fail(SSORT_EINVAL, "null device buffer");
    if (((uintptr_t)d_text & 15) != 0) return fail(SSORT_EINVAL, "text must be 16-byte aligned");
    return with_device(ctx, [&]() -> int {
        ctx->st = stream ? (cudaStream_t)stream : ctx->own_stream;
        int rc = [&]() -> int {
            if (mode == SSORT_TEXT_SUFFIXES) {
                *n_out = text_len;
                SS_TRY(text_fits(text_len, cap));
                LAUNCH(ctx, "iota_offs", launch_iota_offs(d_offs, off_width, text_len, ctx->st));
                return SSORT_OK;
            }
            const uint8_t delim = mode == SSORT_TEXT_LINES ? '\n' : 0;
            uint64_t n = 0;
            SS_TRY(text_count(ctx, d_text, text_len, delim, &n));
            *n_out = n;
            SS_TRY(text_fits(n, cap));
            if (n) SS_TRY(text_write(ctx, d_text, text_len, delim, n, d_offs, off_width));
            return SSORT_OK;
        }();
        ctx->st = ctx->own_stream;
        return rc;
    });
}

int ssort_sort_host_chunked(ssort_ctx *ctx, const uint8_t *arena, uint64_t arena_bytes,
                            const void *offs, int off_width, uint64_t n, uint64_t chunk_strings,
                            uint32_t *perm, uint32_t *lcp) {
    SS_TRY(validate_common(ctx, off_width, n));
    if (n == 0) return SSORT_OK;
    if (!arena || !offs || !perm) return fail(SSORT_EINVAL, "null host buffer");
    if (chunk_strings == 0) return fail(SSORT_EINVAL, "chunk_strings must be positive");
    const uint64_t chunk = std::min<uint64_t>(chunk_strings, n);
    const uint64_t runs = (n + chunk - 1) / chunk;
    std::vector<uint32_t> run_start(runs + 1);
    for (uint64_t r = 0; r <= runs; ++r) run_start[r] = (uint32_t)std::min(n, r * chunk);
    std::vector<uint32_t> own_lcp;
    if (!lcp) {
        own_lcp.resize(n);
        lcp = own_lcp.data();
    }
    int rc = with_device(ctx, [&]() -> int {
        ctx->st = ctx->own_stream;
        SS_TRY(ctx->ensure(ctx->arena, arena_bytes + 16));
        SS_TRY(ctx->ensure(ctx->offs, chunk * off_width));
        SS_TRY(ctx->ensure(ctx->perm, chunk * 8));
        uint8_t *d_arena = (uint8_t *)ctx->arena.p;
        uint32_t *d_perm = (uint32_t *)ctx->perm.p, *d_lcp = d_perm + chunk;
        SS_CUDA(cudaMemcpyAsync(d_arena, arena, arena_bytes, cudaMemcpyHostToDevice, ctx->st));
        SS_CUDA(cudaMemsetAsync(d_arena + arena_bytes, 0, 16, ctx->st));
        for (uint64_t r = 0; r < runs; ++r) {
            const uint64_t lo = run_start[r], m = run_start[r + 1] - lo;
            SS_CUDA(cudaMemcpyAsync(ctx->offs.p, (const uint8_t *)offs + lo * off_width,
                                    m * off_width, cudaMemcpyHostToDevice, ctx->st));
            SS_TRY(sort_device_impl(ctx, d_arena, arena_bytes + 16, ctx->offs.p, off_width, m,
                                    d_perm, d_lcp));
            SS_CUDA(cudaMemcpyAsync(perm + lo, d_perm, m * 4, cudaMemcpyDeviceToHost, ctx->st));
            SS_CUDA(cudaMemcpyAsync(lcp + lo, d_lcp, m * 4, cudaMemcpyDeviceToHost, ctx->st));
        }
        SS_CUDA(cudaStreamSynchronize(ctx->st));
        return SSORT_OK;
    });
    if (rc != SSORT_OK) return rc;
    return ssort_merge_runs(arena, arena_bytes, offs, off_width, n, run_start.data(),
                            (uint32_t)runs, perm, lcp, perm, lcp);
}

int ssort_autotune(ssort_ctx *ctx, const uint8_t *d_arena, uint64_t arena_bytes,
                   const void *d_offs, int off_width, uint64_t n, ssort_tuning *out) {
    SS_TRY(validate_common(ctx, off_width, n));
    if (!out) return fail(SSORT_EINVAL, "null output pointer");
    if (n < 2) return fail(SSORT_EINVAL, "autotuning needs at least 2 strings");
    if (!d_arena || !d_offs) return fail(SSORT_EINVAL, "null device buffer");
    if (((uintptr_t)d_arena & 15) != 0)
        return fail(SSORT_EINVAL, "arena must be 16-byte aligned");
    *out = ssort_tuning{};
    return with_device(ctx, [&]() -> int {
        ctx->st = ctx->own_stream;
        ctx->tuning = true;
        const bool was_prof = ctx->prof;
        ctx->prof = false;
        auto restore = [&]() {
            ctx->tuning = false;
            ctx->prof = was_prof;
        };
        int rc = [&]() -> int {
            SS_TRY(ctx->ensure(ctx->perm, n * 8));
            uint32_t *d_perm = (uint32_t *)ctx->perm.p, *d_lcp = d_perm + n;
            double bits = 0;
            SS_TRY(ctx->sample_entropy(d_arena, arena_bytes, d_offs, off_width, (uint32_t)n,
                                       bits));
            uint32_t trials = 0;
            // Device time of the faster of two sorts under the current values.
            auto time_it = [&](double &ms) -> int {
                ms = 1e30;
                for (int r = 0; r < 2; ++r) {
                    SS_TRY(sort_device_impl(ctx, d_arena, arena_bytes, d_offs, off_width, n,
                                            d_perm, d_lcp));
                    ms = std::min(ms, ctx->stats.device_ms);
                    ++trials;
                }
                return SSORT_OK;
            };
            SS_TRY(sort_device_impl(ctx, d_arena, arena_bytes, d_offs, off_width, n, d_perm,
                                    d_lcp));  // allocations and first-launch costs
            double best = 0;
            SS_TRY(time_it(best));
            const double base = best;
            struct Knob {
                int param;
                std::vector<int64_t> values;
            };
            // Coordinate descent over: range-bucket size, digit width of a
            // partition pass (splitters per pass), the small-segment cutoff,
            // the gather and overlap choices, the CTA sort's record prefetch,
            // the partition's L2 prefetch and the device-driven loop.
            const Knob knobs[] = {{SSORT_PARAM_TARGET_BUCKET, {256, 512, 1024}},
                                  {SSORT_PARAM_DIGIT_BITS, {10, 9, 8}},
                                  {SSORT_PARAM_WARP8_CAP, {64, 128, 256}},
                                  {SSORT_PARAM_FUSED_GATHER, {1, 0}},
                                  {SSORT_PARAM_OVERLAP, {1, 0}},
                                  {SSORT_PARAM_BLOCK_PREFETCH, {1, 0}},
                                  {SSORT_PARAM_L2_PREFETCH, {1, 0}},
                                  {SSORT_PARAM_BLOCK_LEAN, {0, 1, 2}},
                                  {SSORT_PARAM_GRAPH, {0, 1}}};
            auto get = [&](int p) -> int64_t {
                switch (p) {
                    case SSORT_PARAM_TARGET_BUCKET: return ctx->target_bucket;
                    case SSORT_PARAM_DIGIT_BITS: return ctx->digit_bits;
                    case SSORT_PARAM_WARP8_CAP: return ctx->warp8_cap;
                    case SSORT_PARAM_FUSED_GATHER: return ctx->fused_gather;
                    case SSORT_PARAM_BLOCK_PREFETCH: return ctx->block_prefetch ? 1 : 0;
                    case SSORT_PARAM_L2_PREFETCH: return ctx->l2_prefetch ? 1 : 0;
                    case SSORT_PARAM_BLOCK_LEAN: return ctx->block_lean;
                    case SSORT_PARAM_GRAPH: return ctx->graph_mode;
                    default: return ctx->overlap ? 1 : 0;
                }
            };
            for (const Knob &k : knobs) {
                const int64_t start = get(k.param);  // already timed
                int64_t keep = start;
                for (int64_t v : k.values) {
                    if (v == start) continue;
                    SS_TRY(ssort_set_param(ctx, k.param, v));
                    double ms = 0;
                    SS_TRY(time_it(ms));
                    if (ms < best * 0.99) {
                        best = ms;
                        keep = v;
                    }
                }
                SS_TRY(ssort_set_param(ctx, k.param, keep));
            }
            const uint32_t sc = size_class(n), ec = entropy_class(bits);
            ctx->tuned[sc * 4 + ec] = ssort_ctx::Tuned{
                ctx->target_bucket, ctx->warp8_cap, ctx->digit_bits,     ctx->graph_mode,
                ctx->block_lean,    ctx->fused_gather, ctx->overlap,    ctx->block_prefetch,
                ctx->l2_prefetch};
            out->size_class = sc;
            out->entropy_class = ec;
            out->entropy_bits = bits;
            out->target_bucket = ctx->target_bucket;
            out->warp8_cap = ctx->warp8_cap;
            out->overlap = ctx->overlap ? 1 : 0;
            out->fused_gather = ctx->fused_gather;
            out->digit_bits = ctx->digit_bits;
            out->block_prefetch = ctx->block_prefetch ? 1 : 0;
            out->l2_prefetch = ctx->l2_prefetch ? 1 : 0;
            out->graph = ctx->graph_mode;
            out->default_ms = base;
            out->tuned_ms = best;
            out->trials = trials;
            return SSORT_OK;
        }();
        restore();
        return rc;
    });
}

int ssort_pinned_alloc(size_t bytes, void **out) {
    if (!out) return fail(SSORT_EINVAL, "null output pointer");
    *out = nullptr;
    cudaError_t e = cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        cudaGetLastError();
        *out = nullptr;
        return fail(e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? SSORT_ENODEV
                                                                             : SSORT_ENOMEM,
                    std::string("pinned host allocation failed: ") + cudaGetErrorString(e));
    }
    return SSORT_OK;
}

void ssort_pinned_free(void *p) {
    if (p) cudaFreeHost(p);
}

int ssort_sort_text_host(ssort_ctx *ctx, const uint8_t *text, uint64_t text_len, int mode,
                         uint64_t *sorted_offs, uint32_t *lcp, uint64_t cap, uint64_t *n_out) {
    const int w = text_len < (1ull << 32) ? 4 : 8;
    SS_TRY(text_check(ctx, text_len, mode, w, n_out));
    *n_out = 0;
    if (!text_len) return SSORT_OK;
    if (!text) return fail(SSORT_EINVAL, "null text");
    return with_device(ctx, [&]() -> int {
        ctx->st = ctx->own_stream;
        SS_TRY(ctx->ensure(ctx->arena, text_len + 16));
        uint8_t *d_text = (uint8_t *)ctx->arena.p;
        SS_CUDA(cudaMemcpyAsync(d_text, text, text_len, cudaMemcpyHostToDevice, ctx->st));
        SS_CUDA(cudaMemsetAsync(d_text + text_len, 0, 16, ctx->st));
        const uint8_t delim = mode == SSORT_TEXT_LINES ? '\n' : 0;
        uint64_t n = text_len;
        if (mode != SSORT_TEXT_SUFFIXES) SS_TRY(text_count(ctx, d_text, text_len, delim, &n));
        *n_out = n;
        SS_TRY(text_fits(n, cap));
        if (!n) return SSORT_OK;
        if (!sorted_offs) return fail(SSORT_EINVAL, "null output buffer");
        SS_TRY(ctx->ensure(ctx->offs, n * w));
        if (mode == SSORT_TEXT_SUFFIXES)
            LAUNCH(ctx, "iota_offs", launch_iota_offs(ctx->offs.p, w, n, ctx->st));
        else
            SS_TRY(text_write(ctx, d_text, text_len, delim, n, ctx->offs.p, w));
        SS_TRY(ctx->ensure(ctx->perm, n * 4 * (lcp ? 2 : 1)));
        uint32_t *d_perm = (uint32_t *)ctx->perm.p;
        uint32_t *d_lcp = lcp ? d_perm + n : nullptr;
        SS_TRY(sort_device_impl(ctx, d_text, text_len + 16, ctx->offs.p, w, n, d_perm, d_lcp));
        SS_TRY(ctx->ensure(ctx->aux2, n * 8));
        LAUNCH(ctx, "sorted_offs",
               launch_sorted_offs(d_perm, ctx->offs.p, w, n, ctx->aux2.p, 8, ctx->st));
        SS_CUDA(cudaMemcpyAsync(sorted_offs, ctx->aux2.p, n * 8, cudaMemcpyDeviceToHost, ctx->st));
        if (lcp) SS_CUDA(cudaMemcpyAsync(lcp, d_lcp, n * 4, cudaMemcpyDeviceToHost, ctx->st));
        SS_CUDA(cudaStreamSynchronize(ctx->st));
        return SSORT_OK;
    });
}

}  // extern "C"

// ---- sort without device allocation ----------------------------------------
// Some callers cannot let a library call cudaMalloc/cudaFree: cudaFree waits
// for the whole device, allocation can fail or fragment memory that the
// application budgets itself (a server that reserves its device memory up
// front for its own pool, a latency-critical loop that must not block on a
// device-wide synchronisation).  For them the sort's scratch lives in one
// file-scope device array of fixed size, loaded with the library on every
// device that uses it and kept until the process exits.
namespace {

constexpr uint32_t NOALLOC_MAX_N = SSORT_NOALLOC_MAX_N;
constexpr size_t NOALLOC_SCRATCH_BYTES = ws_layout(NOALLOC_MAX_N).total;

// Host code may only name this array to look up its device address; the
// symbol itself is a host-side stand-in, not a device pointer.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

constexpr int NOALLOC_MAX_DEVICES = 64;

struct NoallocDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch
    int num_sms = 0;
    Counters host_ctr{};               // plain host copy of the round counters
};

std::mutex g_noalloc_mu;
NoallocDevice g_noalloc_dev[NOALLOC_MAX_DEVICES];

}  // namespace

extern "C" int ssort_sort_device_noalloc(const uint8_t *d_arena, uint64_t arena_bytes,
                                         const void *d_offs, int off_width, uint64_t n,
                                         uint32_t *d_perm, uint32_t *d_lcp, void *stream) {
    if (off_width != 4 && off_width != 8) return fail(SSORT_EINVAL, "off_width must be 4 or 8");
    if (n > NOALLOC_MAX_N)
        return fail(SSORT_EINVAL, "n = " + std::to_string(n) +
                                      " exceeds the fixed scratch of ssort_sort_device_noalloc (" +
                                      std::to_string(NOALLOC_MAX_N) + " strings)");
    if (n == 0) return SSORT_OK;
    if (!d_arena || !d_offs || !d_perm) return fail(SSORT_EINVAL, "null device buffer");
    if (((uintptr_t)d_arena & 15) != 0)
        return fail(SSORT_EINVAL, "arena must be 16-byte aligned");
    int dev = -1;
    SS_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES) return fail(SSORT_EINVAL, "device index too large");
    // One sort at a time per process: every call shares the scratch array.
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    NoallocDevice &d = g_noalloc_dev[dev];
    if (!d.ready) {
        // First call on this device (with it current): resolve the array's
        // device address.
        void *p = nullptr;
        SS_CUDA(cudaGetSymbolAddress(&p, g_noalloc_scratch));
        SS_CUDA(cudaDeviceGetAttribute(&d.num_sms, cudaDevAttrMultiProcessorCount, dev));
        d.scratch = (unsigned char *)p;
        d.ready = true;
    }
    ssort_ctx c;
    c.device = dev;
    c.num_sms = d.num_sms;
    c.st = (cudaStream_t)stream;
    c.h_ctr = &d.host_ctr;
    c.graph_mode = 0;  // the host-driven loop: building a graph would allocate
    c.ws = ws_bind(ws_layout(NOALLOC_MAX_N), d.scratch);
    c.ws_n = NOALLOC_MAX_N;
    const int rc = c.run_ws(d_arena, arena_bytes, d_offs, off_width, (uint32_t)n, d_perm, d_lcp);
    // Drain the stream on every exit, failed ones included: kernels queued
    // before an error still use the shared scratch, and the next call (which
    // may start as soon as the lock is released) must not race with them.
    const cudaError_t se = cudaStreamSynchronize(c.st);
    c.h_ctr = nullptr;
    if (rc == SSORT_OK && se != cudaSuccess) return cuda_fail(se, "cudaStreamSynchronize");
    return rc;
}
