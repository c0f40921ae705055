// ssort_graph.cu -- the device-driven round loop.
//
// The host round loop (ssort_engine.cu) reads the segment counters back after
// classification, after every partition level and at the end of every round
// to decide the next launches.  Here the same kernels are captured once into
// a CUDA graph whose loops are conditional WHILE nodes (rounds; partition
// levels inside a round) and whose branches are conditional IF nodes (the
// separate key gather of round 0; the count that gathers its own keys on the
// first level of later rounds).  Every kernel finds its work in device
// memory (Count / Span arguments), and small control kernels (k_g_*) advance
// the loop state (GraphState) and set the conditions.  One graph launch runs
// up to GRAPH_ROUNDS_PER_LAUNCH rounds without a host round trip; the host
// reads the state once per launch and relaunches while segments remain.
// Both loops are bounded: a round stops its level loop after max_levels
// levels with an error the host reports, and a launch stops after
// GRAPH_ROUNDS_PER_LAUNCH rounds.
#include "ssort_host.cuh"

#include <cstring>

using namespace ssort;

namespace {

// Adds a conditional node after the current capture dependencies of stream s
// (which is capturing) and makes it the stream's only dependency, so that
// the capture continues after it; returns its body graphs.
int add_conditional(cudaStream_t s, cudaGraphConditionalHandle h,
                    cudaGraphConditionalNodeType type, unsigned size, cudaGraph_t *bodies) {
    cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t *deps = nullptr;
    size_t nd = 0;
    SS_CUDA(cudaStreamGetCaptureInfo(s, &status, nullptr, &g, &deps, &nd));
    if (status != cudaStreamCaptureStatusActive)
        return fail(SSORT_EINTERNAL, "graph build: stream is not capturing");
    cudaGraphNodeParams p{};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = size;
    cudaGraphNode_t node = nullptr;
    SS_CUDA(cudaGraphAddNode(&node, g, deps, nd, &p));
    for (unsigned i = 0; i < size; ++i) bodies[i] = p.conditional.phGraph_out[i];
    SS_CUDA(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    return SSORT_OK;
}

// The bytes that decide a graph's contents: kernel arguments are baked into
// the graph, so a graph is reused only for the same arguments and workspace.
std::vector<unsigned char> graph_key(const SortArgs &a, const ssort_ctx &c) {
    std::vector<unsigned char> k(sizeof(SortArgs) + sizeof(void *) + 2 * sizeof(size_t) + 2);
    unsigned char *p = k.data();
    std::memcpy(p, &a, sizeof(SortArgs));
    p += sizeof(SortArgs);
    std::memcpy(p, &c.ws_buf.p, sizeof(void *));
    p += sizeof(void *);
    std::memcpy(p, &c.ws_n, sizeof(size_t));
    p += sizeof(size_t);
    const size_t sms = (size_t)c.num_sms;
    std::memcpy(p, &sms, sizeof(size_t));
    p += sizeof(size_t);
    p[0] = c.block_prefetch ? 1 : 0;
    p[1] = 0;
    return k;
}

}  // namespace

void ssort_ctx::graph_release() {
    // A build that failed part-way may have left a stream capturing.
    for (cudaStream_t c : cap) {
        cudaStreamCaptureStatus status = cudaStreamCaptureStatusNone;
        if (c && cudaStreamIsCapturing(c, &status) == cudaSuccess &&
            status != cudaStreamCaptureStatusNone) {
            cudaGraph_t partial = nullptr;
            cudaStreamEndCapture(c, &partial);
        }
    }
    cudaGetLastError();
    if (gexec) cudaGraphExecDestroy(gexec);
    if (graph) cudaGraphDestroy(graph);
    gexec = nullptr;
    graph = nullptr;
    gkey.clear();
}

// The on-chip sorts of the list entries appended since the cursors in the
// graph state (device spans), on capture stream s.
int ssort_ctx::graph_small(const SortArgs &a, cudaStream_t s) {
    GraphState *g = ws.gs;
    Counters *dc = ws.ctr;
    Seg *nxt = ws.N;
    LAUNCH(this, "warp1",
           launch_warp1(a, ws.W1, Span{dcount(&g->cur_w1), dcount(&dc->n_w1)}, nxt, dc,
                        grid_for(8), s));
    LAUNCH(this, "warp8",
           launch_warp8(a, ws.W8, Span{dcount(&g->cur_w8), dcount(&dc->n_w8)}, nxt, dc,
                        grid_for(6), s));
    Seg *lists[3] = {ws.S, ws.S2, ws.S3};
    const uint32_t *counts[3] = {&dc->n_small, &dc->n_small2, &dc->n_small3};
    for (int k = 0; k < 3; ++k)
        LAUNCH(this, "block",
               launch_block(a, lists[k], Span{dcount(&g->cur_s[k]), dcount(counts[k])}, k, nxt,
                            dc, grid_for(block_prefetch ? 4 : 6), s, block_prefetch));
    LAUNCH(this, "equal",
           launch_equal(a, ws.E, Span{dcount(&g->cur_e), dcount(&dc->n_equal)}, nxt, dc,
                        grid_for(8), s));
    return SSORT_OK;
}

int ssort_ctx::graph_build(const SortArgs &a) {
    graph_release();
    for (auto &c : cap)
        if (!c) SS_CUDA(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
    GraphState *g = ws.gs;
    Counters *dc = ws.ctr;
    const Count nl = dcount(&g->n_large);
    const int g8 = grid_for(8), g4 = grid_for(4), g2 = grid_for(2);
    const SmallLists S{{ws.S, ws.S2, ws.S3}};
    cudaGraph_t top = nullptr;
    SS_CUDA(cudaGraphCreate(&top, 0));
    graph = top;
    cudaGraphConditionalHandle h_round, h_level, h_gather, h_first;
    SS_CUDA(cudaGraphConditionalHandleCreate(&h_round, top, 1, cudaGraphCondAssignDefault));
    SS_CUDA(cudaGraphConditionalHandleCreate(&h_level, top, 0, cudaGraphCondAssignDefault));
    SS_CUDA(cudaGraphConditionalHandleCreate(&h_gather, top, 0, cudaGraphCondAssignDefault));
    SS_CUDA(cudaGraphConditionalHandleCreate(&h_first, top, 0, cudaGraphCondAssignDefault));
    // The round loop is the graph's only top-level node.
    cudaGraphNodeParams rp{};
    rp.type = cudaGraphNodeTypeConditional;
    rp.conditional.handle = h_round;
    rp.conditional.type = cudaGraphCondTypeWhile;
    rp.conditional.size = 1;
    cudaGraphNode_t rnode = nullptr;
    SS_CUDA(cudaGraphAddNode(&rnode, top, nullptr, 0, &rp));
    cudaGraph_t round_body = rp.conditional.phGraph_out[0];

    cudaStream_t s0 = cap[0], s1 = cap[1], s2 = cap[2];
    const cudaStreamCaptureMode mode = cudaStreamCaptureModeRelaxed;
    cudaGraph_t out = nullptr;
    SS_CUDA(cudaStreamBeginCaptureToGraph(s0, round_body, nullptr, nullptr, 0, mode));
    {
        LAUNCH(this, "g_round_begin", launch_g_round_begin(g, dc, h_round, s0));
        LAUNCH(this, "classify",
               launch_classify(ws.R, dcount(&g->n_cur), a.warp8_cap, ws.W1, ws.W8, S, ws.L, dc,
                               g8, s0));
        LAUNCH(this, "g_after_classify", launch_g_after_classify(g, dc, h_level, h_gather, s0));
        // Round 0 (and rounds without the fused gather): gather the large
        // segments' keys in a separate pass.
        cudaGraph_t gb[1];
        SS_TRY(add_conditional(s0, h_gather, cudaGraphCondTypeIf, 1, gb));
        SS_CUDA(cudaStreamBeginCaptureToGraph(s1, gb[0], nullptr, nullptr, 0, mode));
        LAUNCH(this, "seg_tiles", launch_seg_tiles(ws.L, nl, GATHER_TILE, ws.tile_base, s1));
        LAUNCH(this, "gather", launch_gather(a, ws.L, nl, ws.tile_base, dc, g8, s1));
        SS_CUDA(cudaStreamEndCapture(s1, &out));
        // Partition levels while large segments remain.
        cudaGraph_t lb[1];
        SS_TRY(add_conditional(s0, h_level, cudaGraphCondTypeWhile, 1, lb));
        SS_CUDA(cudaStreamBeginCaptureToGraph(s1, lb[0], nullptr, nullptr, 0, mode));
        {
            LAUNCH(this, "g_level_begin", launch_g_level_begin(g, h_level, h_first, s1));
            cudaGraph_t fb[2];
            SS_TRY(add_conditional(s1, h_first, cudaGraphCondTypeIf, 2, fb));
            for (int f = 0; f < 2; ++f) {
                const bool gather = f == 0;  // body 0 runs when the condition is set
                SS_CUDA(cudaStreamBeginCaptureToGraph(s2, fb[f], nullptr, nullptr, 0, mode));
                LAUNCH(this, "sample",
                       launch_sample(a, ws.L, nl, ws.spl, ws.nspl, ws.tbl, ws.ntiles, ws.cm_size,
                                     gather, g2, s2));
                LAUNCH(this, "scan_pair",
                       launch_scan_pair(ws.ntiles, ws.tile_base, ws.cm_size, ws.cm_base, nl, s2));
                LAUNCH(this, gather ? "count_gather" : "count",
                       launch_count(a, ws.L, nl, ws.tile_base, ws.spl, ws.nspl, ws.tbl,
                                    ws.cm_base, ws.cm, dc, gather, g2, s2));
                SS_CUDA(cudaStreamEndCapture(s2, &out));
            }
            SS_TRY(scan_on(ws.cm, ws.cm, (uint32_t)(ws.cm_cap - 1),
                           dcount(ws.cm_base, &g->n_large), s1));
            LAUNCH(this, "scatter",
                   launch_scatter(a, ws.L, nl, ws.tile_base, ws.spl, ws.nspl, ws.tbl, ws.cm_base,
                                  ws.cm, g2, s1));
            LAUNCH(this, "emit",
                   launch_emit(a, ws.L, nl, ws.tile_base, ws.nspl, ws.cm_base, ws.cm, ws.W1,
                               ws.W8, S, ws.L2, ws.E, ws.B, ws.N, dc, g4, s1));
            SS_TRY(graph_small(a, s1));
            LAUNCH(this, "g_level_end",
                   launch_g_level_end(g, dc, ws.L, ws.L2, h_level, grid_for(1), s1));
        }
        SS_CUDA(cudaStreamEndCapture(s1, &out));
        SS_TRY(graph_small(a, s0));  // what the last level (or classification) left
        LAUNCH(this, "boundary", launch_boundary(a, ws.B, dc, g4, s0));
        LAUNCH(this, "g_round_end", launch_g_round_end(g, dc, ws.R, ws.N, h_round, g2, s0));
    }
    SS_CUDA(cudaStreamEndCapture(s0, &out));
    SS_CUDA(cudaGraphInstantiate(&gexec, top, 0));
    gkey = graph_key(a, *this);
    return SSORT_OK;
}

// Whether this sort runs through the graph: always in mode 1; in mode 2 for
// batched sorts and sorts of at most GRAPH_AUTO_MAX_N strings (where launch
// and host round-trip costs are a large share; large single sorts keep the
// host loop, whose round 0 overlaps the on-chip sorts with the partition on a
// second stream), when a graph for these arguments exists or the previous
// sort had them too.
bool ssort_ctx::graph_wanted(const SortArgs &a, bool batched) {
    if (graph_mode == 1) return true;
    if (!batched && a.n > GRAPH_AUTO_MAX_N) return false;
    std::vector<unsigned char> k = graph_key(a, *this);
    if (!gkey.empty() && k == gkey) return true;
    const bool repeat = k == last_key;
    last_key = std::move(k);
    return repeat;
}

// One sort through the graph: the prologue (identity permutation, the first
// round's segments, the loop state) is launched from the host, then the
// graph runs rounds until none is left.
int ssort_ctx::run_graph(const SortArgs &a, uint32_t n, const uint32_t *d_inst, uint32_t ninst) {
    if (gkey != graph_key(a, *this)) {
        const int rc = graph_build(a);
        if (rc != SSORT_OK) {
            graph_release();
            return rc;
        }
    }
    if (!h_gs) SS_CUDA(cudaHostAlloc((void **)&h_gs, sizeof(GraphState), cudaHostAllocDefault));
    GraphState *g = ws.gs;
    Counters *dc = ws.ctr;
    LAUNCH(this, "iota", launch_iota(a.idx[0], n, st));
    SS_CUDA(cudaMemsetAsync(a.lcp, 0, 4, st));
    std::memset(h_gs, 0, sizeof(GraphState));
    h_gs->fused = fused_gather;
    h_gs->max_levels = graph_max_levels;
    if (d_inst) {
        SS_CUDA(cudaMemcpyAsync(g, h_gs, sizeof(GraphState), cudaMemcpyHostToDevice, st));
        SS_CUDA(cudaMemsetAsync(dc, 0, sizeof(Counters), st));
        LAUNCH(this, "init_batch", launch_init_batch(d_inst, ninst, ws.R, a.lcp, dc, st));
        SS_CUDA(cudaMemcpyAsync(&g->n_cur, &dc->n_next, 4, cudaMemcpyDeviceToDevice, st));
    } else {
        if (n < 2) return SSORT_OK;
        h_gs->n_cur = 1;
        SS_CUDA(cudaMemcpyAsync(g, h_gs, sizeof(GraphState), cudaMemcpyHostToDevice, st));
        const Seg first{0, n, 0, 0};
        SS_CUDA(cudaMemcpyAsync(ws.R, &first, sizeof(Seg), cudaMemcpyHostToDevice, st));
    }
    uint32_t launches = 0;
    for (;; ++launches) {
        // Every launch runs at least one round or ends the sort; a sort needs
        // at most one round per 16 bytes of its longest shared prefix.
        if (launches > (1u << 22))
            return fail(SSORT_EINTERNAL, "device-driven round loop did not finish");
        SS_CUDA(cudaGraphLaunch(gexec, st));
        SS_CUDA(cudaMemcpyAsync(h_gs, g, sizeof(GraphState), cudaMemcpyDeviceToHost, st));
        SS_CUDA(cudaStreamSynchronize(st));
        if (h_gs->error == 2)
            return fail(SSORT_EINTERNAL, "a scan's look-back waited past its bound");
        if (h_gs->error)
            return fail(SSORT_EINTERNAL, "partition levels exceeded " +
                                             std::to_string(graph_max_levels) + " in a round");
        if (h_gs->done || !h_gs->n_cur) break;
        SS_CUDA(cudaMemsetAsync(&g->round_in_launch, 0, 4, st));
    }
    stats.rounds = h_gs->round;
    stats.partition_levels = h_gs->partition_levels;
    for (uint32_t r = 0; r < SSORT_MAX_ROUNDS && r < 64; ++r) stats.live[r] = h_gs->live[r];
    stats.small_segments = h_gs->small_segments;
    stats.partitioned = h_gs->partitioned;
    stats.gather_elems = h_gs->gather_elems;
    stats.gather_fused = h_gs->gather_fused;
    stats.warp1_fresh = h_gs->warp1_fresh;
    stats.warp1_keyed = h_gs->warp1_keyed;
    stats.warp8_fresh = h_gs->warp8_fresh;
    stats.warp8_keyed = h_gs->warp8_keyed;
    stats.block_fresh = h_gs->block_fresh;
    stats.block_keyed = h_gs->block_keyed;
    stats.equal_moved = h_gs->equal_moved;
    stats.equal_final = h_gs->equal_final;
    stats.boundaries = h_gs->boundaries;
    stats.warp1_deep = h_gs->warp1_deep;
    stats.full_sorted = h_gs->full_sorted;
    stats.window_saved = h_gs->window_saved;
    stats.window_used = h_gs->window_used;
    stats.graph_launches = launches + 1;
    if (d_inst) LAUNCH(this, "localize", launch_localize(a.idx[0], n, d_inst, ninst, st));
    return SSORT_OK;
}
