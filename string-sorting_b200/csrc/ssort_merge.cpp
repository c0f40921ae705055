// ssort_merge.cpp -- the consumer side of the LCP array: merging sorted runs
// with their LCPs on the host (ssort_merge_runs), which the chunked sort
// (ssort_sort_host_chunked) uses to sort more strings than one device
// workspace holds.
//
// The merge is the LCP-aware two-way merge of the reference's mergesort_lcp
// (src/mergesort_lcp.cpp:133-211): of the two run heads, the one sharing the
// longer prefix with the last output string is the smaller; only equal LCPs
// need a byte comparison, and it starts at that LCP.  Runs are merged
// pairwise, level by level, with the pairs of one level in parallel.  Ties go
// to the earlier run, so merging runs in input order keeps the sort stable.
#include "ssort_b200.h"

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>
#include <omp.h>

namespace ssort {
int fail(int code, const std::string &msg);
}

namespace {

struct Strings {
    const uint8_t *arena;
    uint64_t bytes;
    const void *offs;
    int width;
    uint64_t start(uint32_t i) const {
        return width == 8 ? static_cast<const uint64_t *>(offs)[i]
                          : static_cast<const uint32_t *>(offs)[i];
    }
    // Bytes at or past the arena end read as NUL, as on the device.
    uint8_t at(uint64_t p) const { return p < bytes ? arena[p] : 0; }
    // (sign of a - b, common prefix length), comparing from depth on.
    std::pair<int, uint32_t> compare(uint32_t a, uint32_t b, uint32_t depth) const {
        const uint64_t pa = start(a), pb = start(b);
        for (uint64_t k = depth;; ++k) {
            const uint8_t x = at(pa + k), y = at(pb + k);
            if (x == 0 || x != y) return {int(x) - int(y), (uint32_t)k};
        }
    }
};

// Merges run 0 (idx0/lcp0, n0 >= 1) and run 1 (n1 >= 1) into out/out_lcp.
// lcp0[i] is the LCP of idx0[i] with idx0[i-1] (lcp0[0]: with whatever
// precedes the run, 0 here); the same for run 1 and for the output.
void merge2(const Strings &s, const uint32_t *idx0, const uint32_t *lcp0, size_t n0,
            const uint32_t *idx1, const uint32_t *lcp1, size_t n1, uint32_t *out,
            uint32_t *out_lcp) {
    size_t i = 0, j = 0, k = 0;
    // h0/h1: LCP of each run's head with the last string written.
    uint32_t h0, h1;
    {
        const auto c = s.compare(idx0[0], idx1[0], 0);
        out_lcp[k] = lcp0[0];
        if (c.first <= 0) {
            out[k++] = idx0[i++];
            h1 = c.second;
            h0 = i < n0 ? lcp0[i] : 0;
        } else {
            out[k++] = idx1[j++];
            h0 = c.second;
            h1 = j < n1 ? lcp1[j] : 0;
        }
    }
    while (i < n0 && j < n1) {
        if (h0 > h1) {
            out[k] = idx0[i];
            out_lcp[k++] = h0;
            ++i;
            h0 = i < n0 ? lcp0[i] : 0;
        } else if (h0 < h1) {
            out[k] = idx1[j];
            out_lcp[k++] = h1;
            ++j;
            h1 = j < n1 ? lcp1[j] : 0;
        } else {
            const auto c = s.compare(idx0[i], idx1[j], h0);
            out_lcp[k] = h0;
            if (c.first <= 0) {
                out[k++] = idx0[i++];
                h1 = c.second;
                h0 = i < n0 ? lcp0[i] : 0;
            } else {
                out[k++] = idx1[j++];
                h0 = c.second;
                h1 = j < n1 ? lcp1[j] : 0;
            }
        }
    }
    for (; i < n0; ++i, ++k) {
        out[k] = idx0[i];
        out_lcp[k] = h0;
        h0 = i + 1 < n0 ? lcp0[i + 1] : 0;
    }
    for (; j < n1; ++j, ++k) {
        out[k] = idx1[j];
        out_lcp[k] = h1;
        h1 = j + 1 < n1 ? lcp1[j + 1] : 0;
    }
}

}  // namespace

extern "C" int ssort_merge_runs(const uint8_t *arena, uint64_t arena_bytes, const void *offs,
                                int off_width, uint64_t n, const uint32_t *run_start,
                                uint32_t nruns, const uint32_t *perm, const uint32_t *lcp,
                                uint32_t *out_perm, uint32_t *out_lcp) {
    using ssort::fail;
    if (off_width != 4 && off_width != 8) return fail(SSORT_EINVAL, "off_width must be 4 or 8");
    if (n > SSORT_MAX_N) return fail(SSORT_EINVAL, "n exceeds SSORT_MAX_N");
    if (n == 0) return SSORT_OK;
    if (!arena || !offs || !run_start || !perm || !lcp || !out_perm || !out_lcp)
        return fail(SSORT_EINVAL, "null buffer");
    if (nruns == 0 || run_start[0] != 0 || run_start[nruns] != n)
        return fail(SSORT_EINVAL, "run table must start at 0 and end at n");
    for (uint32_t r = 0; r < nruns; ++r)
        if (run_start[r + 1] < run_start[r])
            return fail(SSORT_EINVAL, "run table not non-decreasing");
    for (uint32_t r = 0; r < nruns; ++r)
        for (uint32_t p = run_start[r]; p < run_start[r + 1]; ++p)
            if (perm[p] >= run_start[r + 1] - run_start[r])
                return fail(SSORT_EINVAL, "run-local index out of range");
    const Strings s{arena, arena_bytes, offs, off_width};
    // Level 0: run-local indices -> global; every run starts with LCP 0.
    std::vector<uint32_t> ia(n), la(n), ib(n), lb(n);
#pragma omp parallel for schedule(dynamic, 1) if (nruns > 1)
    for (int64_t r = 0; r < (int64_t)nruns; ++r) {
        const uint32_t lo = run_start[r], hi = run_start[r + 1];
        for (uint32_t p = lo; p < hi; ++p) {
            ia[p] = lo + perm[p];
            la[p] = p == lo ? 0 : lcp[p];
        }
    }
    std::vector<uint32_t> bounds(run_start, run_start + nruns + 1);
    bounds.erase(std::unique(bounds.begin(), bounds.end()), bounds.end());  // drop empty runs
    while (bounds.size() > 2) {
        const size_t runs = bounds.size() - 1, pairs = runs / 2;
#pragma omp parallel for schedule(dynamic, 1)
        for (int64_t q = 0; q < (int64_t)pairs; ++q) {
            const uint32_t a = bounds[2 * q], m = bounds[2 * q + 1], b = bounds[2 * q + 2];
            merge2(s, &ia[a], &la[a], m - a, &ia[m], &la[m], b - m, &ib[a], &lb[a]);
        }
        if (runs & 1) {
            const uint32_t a = bounds[runs - 1], b = bounds[runs];
            std::memcpy(&ib[a], &ia[a], (size_t)(b - a) * 4);
            std::memcpy(&lb[a], &la[a], (size_t)(b - a) * 4);
        }
        std::vector<uint32_t> next;
        for (size_t r = 0; r < runs; r += 2) next.push_back(bounds[r]);
        next.push_back(bounds[runs]);
        bounds.swap(next);
        ia.swap(ib);
        la.swap(lb);
    }
    std::memcpy(out_perm, ia.data(), n * 4);
    std::memcpy(out_lcp, la.data(), n * 4);
    return SSORT_OK;
}
