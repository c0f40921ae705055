// ssort_host.cuh -- host-side context shared by the sort engine and the
// request server: the device workspace, the stream the kernels run on, the
// per-kernel profiling records, status helpers and the LAUNCH macro.
#pragma once
#include "ssort_b200.h"
#include "ssort_internal.cuh"

#include <algorithm>
#include <map>
#include <string>
#include <vector>

namespace ssort {

// Records msg as this thread's last error (ssort_last_error) and returns code.
int fail(int code, const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);

struct DBuf {
    void *p = nullptr;
    size_t cap = 0;
};

struct HBuf {
    void *p = nullptr;
    size_t cap = 0;
};

}  // namespace ssort

#define SS_CUDA(call)                                               \
    do {                                                            \
        cudaError_t e_ = (call);                                    \
        if (e_ != cudaSuccess) return ssort::cuda_fail(e_, #call);  \
    } while (0)

#define SS_TRY(call)                   \
    do {                               \
        int r_ = (call);               \
        if (r_ != SSORT_OK) return r_; \
    } while (0)

struct ssort_ctx {
    int device = 0;
    int num_sms = 148;
    cudaStream_t own_stream = nullptr;
    cudaStream_t st = nullptr;
    // The on-chip sorts of a round run on `side` while the partition levels
    // continue on `st` (fork/join through the two events).  Without a side
    // stream, or while profiling, they run on `st`.
    // Within a round the partition levels run on `hp` (forked from and
    // joined back into `st`), the warp sorts and equality buckets on `side`
    // and the CTA sorts on `side2`, all at the default priority, so that the
    // sorts fill the SMs the partition's latency-bound passes leave idle.
    cudaStream_t side = nullptr, side2 = nullptr, hp = nullptr;
    cudaEvent_t ev_fork = nullptr, ev_join = nullptr, ev_join2 = nullptr, ev_round = nullptr;
    bool overlap_round = false;  // this round runs its on-chip sorts on `side`
    bool fresh_round = false;    // this round gathers round-0 style (see round())
    int round_mode = -1;         // -1: fresh iff round_no == 0; 0: fresh; 1: deep

    // workspace
    ssort::DBuf ws_buf;    // one block holding every scratch buffer (ws_layout)
    ssort::Workspace ws{};
    size_t ws_n = 0;  // string capacity ws is laid out for
    ssort::DBuf arena, offs, perm, inst;  // staging for the host-buffer entry points
    ssort::DBuf aux, aux2;  // text inputs: tile counts + scan partials, sorted offsets
    ssort::DBuf key2_buf;   // round-1 keys saved by round 0 (SortArgs::key2)
    ulonglong2 *key2 = nullptr;  // set by run() for the sort it starts
    double round1_live = -1.0;   // share of strings entering round 1 in the last sort
    ssort::HBuf h_offs, h_arena, h_perm;
    // Pinned staging ring for copying pageable host spans to the device
    // (copy_pageable): two chunks, each reused once its transfer is done.
    ssort::HBuf h_stage[2];
    cudaEvent_t ev_stage[2] = {nullptr, nullptr};
    int copy_pageable(void *d_dst, const void *h_src, uint64_t bytes);
    ssort::Counters *h_ctr = nullptr;

    ssort_stats stats{};
    cudaEvent_t ev_start = nullptr, ev_stop = nullptr;

    bool prof = false;
    // tuning parameters (ssort_set_param, ssort_autotune)
    uint32_t target_bucket = ssort::TARGET_BUCKET;  // wanted strings per range bucket
    uint32_t warp8_cap = ssort::WARP8_CAP;          // largest one-warp segment
    uint32_t warp1_deep = ssort::WARP1_DEEP;        // in-warp refinement steps
    bool overlap = true;       // round-0 on-chip sorts on the side stream
    uint32_t fused_gather = 1;  // 1: rounds >= 1 gather inside the first count; 2: all rounds
    bool block_prefetch = false;  // double-buffered CTA sort (k_block2)
    uint32_t block_lean = 0;      // CTA sort: 1 finish from the packed windows, 2 also a
                                  // first sort on 32-bit packed keys
    bool l2_prefetch = false;    // partition kernels prefetch their next tile into L2
    uint32_t digit_bits = 10;    // a partition pass makes at most 2^digit_bits buckets
    uint32_t scatter_variant = 0;  // 1: the scatter stages indices only (k_scatter2)
    bool match_vote = false;       // count kernel ranks keys with ballots
    bool warp_merge = true;        // warp sorts: local networks + merge passes
    bool scan_lookback = true;     // count-matrix scan in one pass (decoupled look-back)
    // Device-driven round loop (ssort_graph.cu): the instantiated graph, the
    // key it was built for, three streams to capture nested conditional
    // bodies on, and a pinned copy of the loop state.
    // 0 (default): host loop; 1: device-driven loop always; 2 (auto): the
    // device-driven loop for batched sorts and sorts of at most
    // GRAPH_AUTO_MAX_N strings, once a sort repeats the previous sort's
    // arguments (buffers, size, workspace), since building a graph costs more
    // than one host-driven sort
    uint32_t graph_mode = 0;
    std::vector<unsigned char> last_key;  // arguments of the previous sort (auto mode)
    uint32_t graph_max_levels = ssort::GRAPH_MAX_LEVELS;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t gexec = nullptr;
    std::vector<unsigned char> gkey;
    cudaStream_t cap[3] = {nullptr, nullptr, nullptr};
    ssort::GraphState *h_gs = nullptr;
    // Autotuned values per (size class * 4 + entropy class), applied to later
    // sorts of the same classes; not while the tuner itself runs.
    struct Tuned {
        uint32_t target_bucket, warp8_cap, digit_bits, graph, block_lean, fused_gather;
        bool overlap, block_prefetch, l2_prefetch;
    };
    std::map<uint32_t, Tuned> tuned;
    // target buckets per segment size class for the next batched sort
    // (SortArgs::target_by_class), from the tuned entries of each class
    uint16_t class_targets[32] = {};
    bool tuning = false;
    ssort::DBuf hist_buf;
    uint32_t *h_hist = nullptr;
    int sample_entropy(const uint8_t *arena, uint64_t arena_bytes, const void *offs,
                       int off_width, uint32_t n, double &bits);
    struct Rec {
        const char *name;
        cudaEvent_t a, b;
    };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> ev_pool;
    size_t ev_used = 0;
    std::map<std::string, std::pair<double, uint64_t>> ktimes;

    int ensure(ssort::DBuf &b, size_t bytes) {
        if (b.cap >= bytes) return SSORT_OK;
        if (b.p) cudaFree(b.p);
        b.p = nullptr;
        b.cap = 0;
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&b.p, want);
        if (e != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return ssort::fail(SSORT_ENOMEM, "device allocation of " + std::to_string(want) +
                                          " bytes failed: " + cudaGetErrorString(e));
        }
        b.cap = want;
        return SSORT_OK;
    }

    int ensure_host(ssort::HBuf &b, size_t bytes) {
        if (b.cap >= bytes) return SSORT_OK;
        if (b.p) cudaFreeHost(b.p);
        b.p = nullptr;
        b.cap = 0;
        cudaError_t e = cudaHostAlloc(&b.p, std::max<size_t>(bytes, 256), cudaHostAllocDefault);
        if (e != cudaSuccess) {
            cudaGetLastError();
            b.p = nullptr;
            return ssort::fail(SSORT_ENOMEM, "pinned host allocation failed");
        }
        b.cap = std::max<size_t>(bytes, 256);
        return SSORT_OK;
    }

    cudaEvent_t pool_event() {
        if (ev_used == ev_pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            ev_pool.push_back(e);
        }
        return ev_pool[ev_used++];
    }

    void prof_begin(const char *name) {
        if (!prof) return;
        Rec r{name, pool_event(), pool_event()};
        cudaEventRecord(r.a, st);
        recs.push_back(r);
    }
    void prof_end() {
        if (!prof) return;
        cudaEventRecord(recs.back().b, st);
    }
    void prof_collect() {
        for (auto &r : recs) {
            float ms = 0;
            cudaEventElapsedTime(&ms, r.a, r.b);
            auto &slot = ktimes[r.name];
            slot.first += ms;
            slot.second += 1;
        }
        recs.clear();
        ev_used = 0;
    }

    int check_launch(const char *name) {
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return ssort::cuda_fail(e, name);
        return SSORT_OK;
    }

    int sync_counters() {
        SS_CUDA(cudaMemcpyAsync(h_ctr, ws.ctr, sizeof(ssort::Counters), cudaMemcpyDeviceToHost, st));
        SS_CUDA(cudaStreamSynchronize(st));
        if (h_ctr->error)
            return ssort::fail(SSORT_EINTERNAL, "a scan's look-back waited past its bound");
        return SSORT_OK;
    }

    int grid_for(int per_sm) const { return num_sms * per_sm; }

    int reserve(uint32_t n);
    int scan(const uint32_t *in, uint32_t *out, uint32_t cap, ssort::Count n);
    int scan_on(const uint32_t *in, uint32_t *out, uint32_t cap, ssort::Count n, cudaStream_t s);
    int run(const uint8_t *arena, uint64_t arena_bytes, const void *offs, int off_width,
            uint32_t n, uint32_t *d_perm, uint32_t *d_lcp, const uint32_t *d_inst = nullptr,
            uint32_t ninst = 0);
    // List entries of the on-chip sorts already launched in this round.
    struct SmallDone {
        uint32_t w1 = 0, w8 = 0, s[3] = {0, 0, 0}, e = 0;
    };
    int fork_small();
    int launch_small(const ssort::SortArgs &a, ssort::Seg *nxt, SmallDone &done);
    int round_body(const ssort::SortArgs &a, ssort::Seg *cur, uint32_t n_cur, ssort::Seg *nxt,
                   uint32_t &n_next, uint32_t round_no);
    int round(const ssort::SortArgs &a, ssort::Seg *cur, uint32_t n_cur, ssort::Seg *nxt,
              uint32_t &n_next,
              uint32_t round_no);
    int run_ws(const uint8_t *arena, uint64_t arena_bytes, const void *offs, int off_width,
               uint32_t n, uint32_t *d_perm, uint32_t *d_lcp, const uint32_t *d_inst = nullptr,
               uint32_t ninst = 0);
    // device-driven round loop (ssort_graph.cu)
    int run_graph(const ssort::SortArgs &a, uint32_t n, const uint32_t *d_inst, uint32_t ninst);
    bool graph_wanted(const ssort::SortArgs &a, bool batched);
    int graph_build(const ssort::SortArgs &a);
    int graph_small(const ssort::SortArgs &a, cudaStream_t s);
    void graph_release();
};

#define LAUNCH(ctx, name, call)                 \
    do {                                        \
        (ctx)->prof_begin(name);                \
        call;                                   \
        (ctx)->prof_end();                      \
        SS_TRY((ctx)->check_launch(name));      \
    } while (0)


// Run fn with the context's device current, restoring the caller's device.
template <class F>
inline int with_device(ssort_ctx *ctx, F fn) {
    int prev = -1;
    cudaGetDevice(&prev);
    if (prev != ctx->device) cudaSetDevice(ctx->device);
    int rc = fn();
    if (prev >= 0 && prev != ctx->device) cudaSetDevice(prev);
    return rc;
}

