// ssort_server.cu -- the request server: continuous batching of independent
// sort requests at round granularity (ssort_server_* in include/ssort_b200.h).
//
// Device state, allocated once at creation and resident for the server's
// life:
//   pool    arena_budget bytes; each admitted request's strings are copied
//           into a first-fit region of it (aligned to 256, one byte longer
//           than the request's arena for a terminating NUL).
//   goffs   uint64 offset into the pool per position.
//   perm    final index per position (the sort's idx[0]).
//   ws      the sort workspace laid out for max_strings positions; its lcp
//           array is the server's lcp output and the staging area for
//           uint32 offsets.
// Each admitted request holds a first-fit range of positions.  Between
// rounds, requests whose copies have landed join the running segment list
// as one depth-0 segment each; one round then refines the segments of every
// joined request together.  After the round, a request that owns no segment
// of the next round is finished: its indices are made request-local and
// copied out on a second copy stream, and its pool region and positions are
// released once that copy has completed.  Segments never span two requests
// and every kernel works per segment, so a request's result does not depend
// on what it shared the rounds with.
#include "ssort_host.cuh"

#include <deque>
#include <mutex>
#include <unordered_map>

using namespace ssort;

namespace {

// First-fit allocator over [0, cap) with coalescing of freed ranges.
class RangeAlloc {
   public:
    void init(uint64_t cap) {
        free_.clear();
        if (cap) free_[0] = cap;
        cap_ = cap;
        used_ = 0;
    }
    bool alloc(uint64_t size, uint64_t align, uint64_t &off) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            const uint64_t start = (it->first + align - 1) / align * align;
            const uint64_t end = it->first + it->second;
            if (start > end || end - start < size) continue;
            const uint64_t lo = it->first, hi = end;
            free_.erase(it);
            if (start > lo) free_[lo] = start - lo;
            if (hi > start + size) free_[start + size] = hi - (start + size);
            off = start;
            used_ += size;
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t size) {
        if (!size) return;
        used_ -= size;
        auto next = free_.lower_bound(off);
        if (next != free_.end() && next->first == off + size) {
            size += next->second;
            next = free_.erase(next);
        }
        if (next != free_.begin()) {
            auto prev = std::prev(next);
            if (prev->first + prev->second == off) {
                prev->second += size;
                return;
            }
        }
        free_[off] = size;
    }
    uint64_t used() const { return used_; }

   private:
    std::map<uint64_t, uint64_t> free_;
    uint64_t cap_ = 0, used_ = 0;
};

constexpr uint64_t REGION_ALIGN = 256;
constexpr uint32_t MAX_SLOTS = 1u << 16;  // requests held on the device at once

uint64_t region_bytes(uint64_t arena_bytes) {
    return (arena_bytes + 1 + REGION_ALIGN - 1) / REGION_ALIGN * REGION_ALIGN;
}

struct Request {
    uint64_t id = 0;
    const uint8_t *arena = nullptr;
    uint64_t arena_bytes = 0;
    const void *offs = nullptr;
    int off_width = 8;
    uint32_t n = 0;
    uint32_t *perm_out = nullptr, *lcp_out = nullptr;
    int state = SSORT_REQ_QUEUED;
    uint64_t region = 0, region_size = 0;
    uint64_t pos = 0;
    cudaEvent_t ev = nullptr;  // copy-in done, then copy-out done
};

}  // namespace

struct ssort_server {
    std::mutex mu;
    ssort_ctx *ctx = nullptr;  // compute stream, workspace, kernels
    cudaStream_t h2d = nullptr, d2h = nullptr;  // copy-in and copy-out streams
    uint64_t budget = 0;
    uint32_t max_strings = 0;
    DBuf pool, goffs, perm, bases, flags, d_join, d_done;
    uint32_t *h_bases = nullptr, *h_flags = nullptr;
    ReqJob *h_join = nullptr, *h_done = nullptr;  // pinned job tables
    cudaEvent_t ev_join_jobs = nullptr, ev_done_jobs = nullptr, ev_unbased = nullptr;
    bool join_jobs_pending = false, done_jobs_pending = false;
    RangeAlloc arena_alloc, pos_alloc;
    std::deque<Request *> queue;
    std::vector<Request *> loading, active, draining;
    std::unordered_map<uint64_t, Request *> by_id;
    std::deque<uint64_t> done_ids;
    std::vector<cudaEvent_t> spare_events;
    uint64_t next_id = 1;
    Seg *cur = nullptr, *nxt = nullptr;
    uint32_t n_cur = 0;
    uint64_t rounds = 0, requests_done = 0, strings_done = 0;
    uint64_t joined_strings = 0;  // strings joined in this step
    uint64_t prev_live = 0;       // strings live in the last round
    uint32_t max_active = 0;
    int error = SSORT_OK;
    std::string error_msg;

    cudaEvent_t take_event() {
        if (!spare_events.empty()) {
            cudaEvent_t e = spare_events.back();
            spare_events.pop_back();
            return e;
        }
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        return e;
    }
    void give_event(cudaEvent_t e) {
        if (e) spare_events.push_back(e);
    }

    SortArgs args() const {
        SortArgs a{};
        a.arena = (const uint8_t *)pool.p;
        a.arena_bytes = budget;
        a.offs = goffs.p;
        a.off_width = 8;
        a.n = max_strings;
        a.idx[0] = (uint32_t *)perm.p;
        a.idx[1] = ctx->ws.idx1;
        a.key[0] = ctx->ws.key0;
        a.key[1] = ctx->ws.key1;
        a.lcp = ctx->ws.lcp;
        a.bkt = ctx->ws.bkt;
        a.target_bucket = ctx->target_bucket;
        a.warp8_cap = ctx->warp8_cap;
        a.warp1_deep = ctx->warp1_deep;
        a.l2_prefetch = ctx->l2_prefetch ? 1u : 0u;
        a.scatter_staged_idx = ctx->scatter_variant;
        a.block_lean = ctx->block_lean;
        a.match_vote = ctx->match_vote ? 1u : 0u;
        a.warp_merge = ctx->warp_merge ? 1u : 0u;
        a.max_splitters = (1u << (ctx->digit_bits - 1)) - 1;
        return a;
    }

    int admit();
    int join();
    int finish(const std::vector<Request *> &done);
    int detect();
    int retire();
    int step_locked();
    int sticky(int rc) {
        if (rc != SSORT_OK && error == SSORT_OK) {
            error = rc;
            error_msg = ssort_last_error();
        }
        return rc;
    }
};

// FIFO admission: the head of the queue is admitted when its pool region and
// position range fit; later requests wait behind it.
int ssort_server::admit() {
    while (!queue.empty()) {
        Request *r = queue.front();
        if (loading.size() + active.size() + draining.size() >= MAX_SLOTS) break;
        uint64_t region = 0, pos = 0;
        const uint64_t rsz = region_bytes(r->arena_bytes);
        if (!arena_alloc.alloc(rsz, REGION_ALIGN, region)) break;
        if (!pos_alloc.alloc(r->n, 1, pos)) {
            arena_alloc.release(region, rsz);
            break;
        }
        queue.pop_front();
        r->region = region;
        r->region_size = rsz;
        r->pos = pos;
        r->ev = take_event();
        if (!r->ev) return fail(SSORT_ECUDA, "event creation failed");
        uint8_t *dst = (uint8_t *)pool.p + region;
        if (r->arena_bytes)
            SS_CUDA(cudaMemcpyAsync(dst, r->arena, r->arena_bytes, cudaMemcpyDefault, h2d));
        SS_CUDA(cudaMemsetAsync(dst + r->arena_bytes, 0, rsz - r->arena_bytes, h2d));
        void *odst = r->off_width == 8 ? (void *)((uint64_t *)goffs.p + pos)
                                       : (void *)(ctx->ws.lcp + pos);
        SS_CUDA(cudaMemcpyAsync(odst, r->offs, (size_t)r->n * r->off_width, cudaMemcpyDefault,
                                h2d));
        SS_CUDA(cudaEventRecord(r->ev, h2d));
        r->state = SSORT_REQ_LOADING;
        loading.push_back(r);
    }
    return SSORT_OK;
}

// Waits until the previous host-to-device copy out of a job table has run,
// so that the pinned table can be refilled.
static int jobs_free(cudaEvent_t ev, bool &pending) {
    if (pending) SS_CUDA(cudaEventSynchronize(ev));
    pending = false;
    return SSORT_OK;
}

// Requests whose copies have landed join the segment list (one launch for
// all of them); with no round in progress every loading request joins and
// the compute stream waits for its copies.
int ssort_server::join() {
    const bool idle = n_cur == 0 && active.empty();
    std::vector<Request *> still, joined;
    for (Request *r : loading) {
        cudaError_t q = cudaEventQuery(r->ev);
        if (q != cudaSuccess && q != cudaErrorNotReady) return cuda_fail(q, "copy-in event");
        if (q == cudaErrorNotReady && !idle) {
            still.push_back(r);
            continue;
        }
        SS_CUDA(cudaStreamWaitEvent(ctx->st, r->ev, 0));
        joined.push_back(r);
    }
    loading.swap(still);
    if (joined.empty()) return SSORT_OK;
    SS_TRY(jobs_free(ev_join_jobs, join_jobs_pending));
    uint32_t total = 0;
    for (size_t k = 0; k < joined.size(); ++k) {
        Request *r = joined[k];
        ReqJob &jb = h_join[k];
        jb.region_base = r->region;
        jb.arena_bytes = r->arena_bytes;
        jb.pos = (uint32_t)r->pos;
        jb.n = r->n;
        jb.first = total;
        jb.slot = r->n >= 2 ? n_cur++ : 0u;
        jb.off_width = (uint32_t)r->off_width;
        jb.pad = 0;
        total += r->n;
        joined_strings += r->n;
        r->state = SSORT_REQ_ACTIVE;
        active.push_back(r);
    }
    const uint32_t nj = (uint32_t)joined.size();
    SS_CUDA(cudaMemcpyAsync(d_join.p, h_join, nj * sizeof(ReqJob), cudaMemcpyHostToDevice,
                            ctx->st));
    SS_CUDA(cudaEventRecord(ev_join_jobs, ctx->st));
    join_jobs_pending = true;
    LAUNCH(ctx, "join",
           launch_join((uint64_t *)goffs.p, ctx->ws.lcp, (uint32_t *)perm.p,
                       (const ReqJob *)d_join.p, nj, total, cur, ctx->st));
    max_active = std::max<uint32_t>(max_active, (uint32_t)active.size());
    return SSORT_OK;
}

// Request-local indices for all finished requests (one launch), then each
// request's copy-out on the device-to-host stream.
int ssort_server::finish(const std::vector<Request *> &done) {
    if (done.empty()) return SSORT_OK;
    SS_TRY(jobs_free(ev_done_jobs, done_jobs_pending));
    uint32_t total = 0;
    for (size_t k = 0; k < done.size(); ++k) {
        ReqJob &jb = h_done[k];
        jb = ReqJob{};
        jb.pos = (uint32_t)done[k]->pos;
        jb.n = done[k]->n;
        jb.first = total;
        total += done[k]->n;
    }
    const uint32_t nd = (uint32_t)done.size();
    SS_CUDA(cudaMemcpyAsync(d_done.p, h_done, nd * sizeof(ReqJob), cudaMemcpyHostToDevice,
                            ctx->st));
    SS_CUDA(cudaEventRecord(ev_done_jobs, ctx->st));
    done_jobs_pending = true;
    LAUNCH(ctx, "unbase",
           launch_unbase((uint32_t *)perm.p, (const ReqJob *)d_done.p, nd, total, ctx->st));
    SS_CUDA(cudaEventRecord(ev_unbased, ctx->st));
    SS_CUDA(cudaStreamWaitEvent(d2h, ev_unbased, 0));
    for (Request *r : done) {
        if (r->n) {
            SS_CUDA(cudaMemcpyAsync(r->perm_out, (uint32_t *)perm.p + r->pos, (size_t)r->n * 4,
                                    cudaMemcpyDefault, d2h));
            if (r->lcp_out)
                SS_CUDA(cudaMemcpyAsync(r->lcp_out, ctx->ws.lcp + r->pos, (size_t)r->n * 4,
                                        cudaMemcpyDefault, d2h));
        }
        SS_CUDA(cudaEventRecord(r->ev, d2h));
        r->state = SSORT_REQ_DRAINING;
        draining.push_back(r);
    }
    return SSORT_OK;
}

// After a round: every joined request that owns no segment of the next round
// is finished.
int ssort_server::detect() {
    if (active.empty()) return SSORT_OK;
    std::vector<Request *> done, keep;
    if (n_cur == 0) {
        done.swap(active);
    } else {
        std::sort(active.begin(), active.end(),
                  [](const Request *x, const Request *y) { return x->pos < y->pos; });
        const uint32_t nact = (uint32_t)active.size();
        for (uint32_t j = 0; j < nact; ++j) h_bases[j] = (uint32_t)active[j]->pos;
        SS_CUDA(cudaMemcpyAsync(bases.p, h_bases, nact * 4, cudaMemcpyHostToDevice, ctx->st));
        SS_CUDA(cudaMemsetAsync(flags.p, 0, nact * 4, ctx->st));
        LAUNCH(ctx, "mark",
               launch_mark(cur, n_cur, (const uint32_t *)bases.p, nact, (uint32_t *)flags.p,
                           ctx->st));
        SS_CUDA(cudaMemcpyAsync(h_flags, flags.p, nact * 4, cudaMemcpyDeviceToHost, ctx->st));
        SS_CUDA(cudaStreamSynchronize(ctx->st));
        for (uint32_t j = 0; j < nact; ++j) (h_flags[j] ? keep : done).push_back(active[j]);
        active.swap(keep);
    }
    return finish(done);
}

// Requests whose copy-out has completed release their pool region and
// positions and are reported done.
int ssort_server::retire() {
    std::vector<Request *> still;
    for (Request *r : draining) {
        cudaError_t q = cudaEventQuery(r->ev);
        if (q == cudaErrorNotReady) {
            still.push_back(r);
            continue;
        }
        if (q != cudaSuccess) return cuda_fail(q, "copy-out event");
        arena_alloc.release(r->region, r->region_size);
        pos_alloc.release(r->pos, r->n);
        give_event(r->ev);
        done_ids.push_back(r->id);
        ++requests_done;
        strings_done += r->n;
        by_id.erase(r->id);
        delete r;
    }
    draining.swap(still);
    return SSORT_OK;
}

int ssort_server::step_locked() {
    SS_TRY(retire());
    SS_TRY(admit());
    joined_strings = 0;
    SS_TRY(join());
    if (n_cur) {
        uint32_t n_next = 0;
        // Mostly newly joined strings (identity indices, request bytes laid
        // out in order in the pool): a fresh round; else a deep one.
        ctx->round_mode = joined_strings * 2 >= prev_live ? 0 : 1;
        SS_TRY(ctx->round(args(), cur, n_cur, nxt, n_next, (uint32_t)std::min<uint64_t>(
                                                                rounds, UINT32_MAX)));
        prev_live = ctx->h_ctr->live_next;
        std::swap(cur, nxt);
        n_cur = n_next;
        ++rounds;
    }
    SS_TRY(detect());
    return SSORT_OK;
}

namespace {

int server_error(ssort_server *srv) {
    return fail(srv->error, "server failed earlier: " + srv->error_msg);
}

void server_free(ssort_server *srv) {
    if (srv->ctx) {
        with_device(srv->ctx, [&]() -> int {
            if (srv->h2d) cudaStreamSynchronize(srv->h2d);
            if (srv->d2h) cudaStreamSynchronize(srv->d2h);
            cudaStreamSynchronize(srv->ctx->st);
            for (DBuf *b : {&srv->pool, &srv->goffs, &srv->perm, &srv->bases, &srv->flags,
                            &srv->d_join, &srv->d_done})
                if (b->p) cudaFree(b->p);
            if (srv->h_bases) cudaFreeHost(srv->h_bases);
            if (srv->h_flags) cudaFreeHost(srv->h_flags);
            if (srv->h_join) cudaFreeHost(srv->h_join);
            if (srv->h_done) cudaFreeHost(srv->h_done);
            for (cudaEvent_t e : {srv->ev_join_jobs, srv->ev_done_jobs, srv->ev_unbased})
                if (e) cudaEventDestroy(e);
            for (auto &kv : srv->by_id) {
                if (kv.second->ev) cudaEventDestroy(kv.second->ev);
                delete kv.second;
            }
            for (auto e : srv->spare_events) cudaEventDestroy(e);
            if (srv->h2d) cudaStreamDestroy(srv->h2d);
            if (srv->d2h) cudaStreamDestroy(srv->d2h);
            return SSORT_OK;
        });
        ssort_ctx_destroy(srv->ctx);
    }
    delete srv;
}

}  // namespace

extern "C" {

int ssort_server_create(int device, uint64_t arena_budget_bytes, uint64_t max_strings,
                        ssort_server **out) {
    if (!out) return fail(SSORT_EINVAL, "null output pointer");
    *out = nullptr;
    if (max_strings == 0 || max_strings > SSORT_MAX_N)
        return fail(SSORT_EINVAL, "max_strings must be in [1, SSORT_MAX_N]");
    if (arena_budget_bytes < REGION_ALIGN)
        return fail(SSORT_EINVAL, "arena budget below 256 bytes");
    ssort_ctx *ctx = nullptr;
    SS_TRY(ssort_ctx_create(device, &ctx));
    ssort_server *srv = new ssort_server();
    srv->ctx = ctx;
    srv->budget = arena_budget_bytes / REGION_ALIGN * REGION_ALIGN;
    srv->max_strings = (uint32_t)max_strings;
    int rc = with_device(ctx, [&]() -> int {
        SS_CUDA(cudaStreamCreateWithFlags(&srv->h2d, cudaStreamNonBlocking));
        SS_CUDA(cudaStreamCreateWithFlags(&srv->d2h, cudaStreamNonBlocking));
        SS_TRY(ctx->reserve(srv->max_strings));
        SS_TRY(ctx->ensure(srv->pool, srv->budget));
        SS_TRY(ctx->ensure(srv->goffs, (size_t)srv->max_strings * 8));
        SS_TRY(ctx->ensure(srv->perm, (size_t)srv->max_strings * 4));
        SS_TRY(ctx->ensure(srv->bases, (size_t)MAX_SLOTS * 4));
        SS_TRY(ctx->ensure(srv->flags, (size_t)MAX_SLOTS * 4));
        SS_CUDA(cudaHostAlloc((void **)&srv->h_bases, (size_t)MAX_SLOTS * 4, cudaHostAllocDefault));
        SS_CUDA(cudaHostAlloc((void **)&srv->h_flags, (size_t)MAX_SLOTS * 4, cudaHostAllocDefault));
        SS_TRY(ctx->ensure(srv->d_join, (size_t)MAX_SLOTS * sizeof(ReqJob)));
        SS_TRY(ctx->ensure(srv->d_done, (size_t)MAX_SLOTS * sizeof(ReqJob)));
        SS_CUDA(cudaHostAlloc((void **)&srv->h_join, (size_t)MAX_SLOTS * sizeof(ReqJob),
                              cudaHostAllocDefault));
        SS_CUDA(cudaHostAlloc((void **)&srv->h_done, (size_t)MAX_SLOTS * sizeof(ReqJob),
                              cudaHostAllocDefault));
        SS_CUDA(cudaEventCreateWithFlags(&srv->ev_join_jobs, cudaEventDisableTiming));
        SS_CUDA(cudaEventCreateWithFlags(&srv->ev_done_jobs, cudaEventDisableTiming));
        SS_CUDA(cudaEventCreateWithFlags(&srv->ev_unbased, cudaEventDisableTiming));
        return SSORT_OK;
    });
    if (rc != SSORT_OK) {
        server_free(srv);
        return rc;
    }
    srv->arena_alloc.init(srv->budget);
    srv->pos_alloc.init(srv->max_strings);
    srv->cur = ctx->ws.R;
    srv->nxt = ctx->ws.N;
    *out = srv;
    return SSORT_OK;
}

void ssort_server_destroy(ssort_server *srv) {
    if (srv) server_free(srv);
}

int ssort_server_submit(ssort_server *srv, const uint8_t *arena, uint64_t arena_bytes,
                        const void *offs, int off_width, uint64_t n, uint32_t *perm_out,
                        uint32_t *lcp_out, uint64_t *id_out) {
    if (!srv || !id_out) return fail(SSORT_EINVAL, "null server or id pointer");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->error) return server_error(srv);
    if (off_width != 4 && off_width != 8) return fail(SSORT_EINVAL, "off_width must be 4 or 8");
    if (n > SSORT_MAX_N) return fail(SSORT_EINVAL, "n exceeds SSORT_MAX_N");
    if (n && (!arena || !offs || !perm_out)) return fail(SSORT_EINVAL, "null host buffer");
    if (n > srv->max_strings || region_bytes(arena_bytes) > srv->budget)
        return fail(SSORT_ENOMEM, "request larger than the server's capacity (" +
                                      std::to_string(n) + " strings, " +
                                      std::to_string(arena_bytes) + " arena bytes)");
    Request *r = new Request();
    r->id = srv->next_id++;
    r->arena = arena;
    r->arena_bytes = arena_bytes;
    r->offs = offs;
    r->off_width = off_width;
    r->n = (uint32_t)n;
    r->perm_out = perm_out;
    r->lcp_out = lcp_out;
    *id_out = r->id;
    if (n == 0) {
        srv->done_ids.push_back(r->id);
        ++srv->requests_done;
        delete r;
        return SSORT_OK;
    }
    srv->by_id[r->id] = r;
    srv->queue.push_back(r);
    return SSORT_OK;
}

int ssort_server_step(ssort_server *srv, uint64_t *done_ids, uint32_t cap, uint32_t *n_done) {
    if (!srv) return fail(SSORT_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->error) return server_error(srv);
    int rc = with_device(srv->ctx, [&]() -> int { return srv->sticky(srv->step_locked()); });
    uint32_t k = 0;
    while (k < cap && done_ids && !srv->done_ids.empty()) {
        done_ids[k++] = srv->done_ids.front();
        srv->done_ids.pop_front();
    }
    if (n_done) *n_done = k;
    return rc;
}

int ssort_server_poll(ssort_server *srv, uint64_t id, int *state) {
    if (!srv || !state) return fail(SSORT_EINVAL, "null server or state pointer");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (id == 0 || id >= srv->next_id) return fail(SSORT_EINVAL, "unknown request id");
    auto it = srv->by_id.find(id);
    *state = it == srv->by_id.end() ? SSORT_REQ_DONE : it->second->state;
    return SSORT_OK;
}

int ssort_server_drain(ssort_server *srv) {
    if (!srv) return fail(SSORT_EINVAL, "null server");
    std::lock_guard<std::mutex> lk(srv->mu);
    if (srv->error) return server_error(srv);
    return with_device(srv->ctx, [&]() -> int {
        while (!srv->by_id.empty()) {
            SS_TRY(srv->sticky(srv->step_locked()));
            if (srv->queue.empty() && srv->loading.empty() && srv->active.empty() &&
                !srv->draining.empty())
                SS_CUDA(cudaEventSynchronize(srv->draining.front()->ev));
        }
        return SSORT_OK;
    });
}

int ssort_server_get_info(ssort_server *srv, ssort_server_info *out) {
    if (!srv || !out) return fail(SSORT_EINVAL, "null server or output pointer");
    std::lock_guard<std::mutex> lk(srv->mu);
    ssort_server_info i{};
    i.queued = (uint32_t)srv->queue.size();
    i.loading = (uint32_t)srv->loading.size();
    i.active = (uint32_t)srv->active.size();
    i.draining = (uint32_t)srv->draining.size();
    i.max_active = srv->max_active;
    i.rounds = srv->rounds;
    i.requests_done = srv->requests_done;
    i.strings_done = srv->strings_done;
    i.arena_in_use = srv->arena_alloc.used();
    i.strings_in_use = srv->pos_alloc.used();
    i.arena_budget = srv->budget;
    i.max_strings = srv->max_strings;
    size_t held = srv->ctx->ws_buf.cap;
    for (DBuf *b : {&srv->pool, &srv->goffs, &srv->perm, &srv->bases, &srv->flags, &srv->d_join,
                    &srv->d_done})
        held += b->cap;
    i.device_bytes = held;
    *out = i;
    return SSORT_OK;
}

}  // extern "C"
