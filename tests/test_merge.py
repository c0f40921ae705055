"""LCP consumers: the host LCP merge of sorted runs (ssort_merge_runs, the
reference's mergesort_lcp two-way merge, src/mergesort_lcp.cpp:133-211) and
the chunked sort built on it.  The merge is host code, so its tests run on
the CPU with runs sorted by the oracle; the merged result must be the oracle's
sort of the whole input, permutation and LCP array alike."""
import hashlib

import numpy as np
import pytest

import cases
import pyoracle
import pyssort


def _runs_by_oracle(arena, offs, run_start):
    perm = np.empty(len(offs), dtype=np.uint32)
    lcp = np.empty(len(offs), dtype=np.uint32)
    for r in range(len(run_start) - 1):
        lo, hi = int(run_start[r]), int(run_start[r + 1])
        if hi > lo:
            perm[lo:hi], lcp[lo:hi] = pyoracle.oracle_sort(arena, offs[lo:hi])
    return perm, lcp


def _cuts(n, k, seed):
    rng = np.random.default_rng(seed)
    inner = np.sort(rng.integers(0, n + 1, size=k - 1))
    return np.concatenate([[0], inner, [n]]).astype(np.uint32)


@pytest.mark.parametrize("name", ["desc_numbers_200000", "long_prefix_10000", "ff_runs_3000",
                                  "high_bytes_5000", "all_empty_100", "ut_aaa_1801"])
@pytest.mark.parametrize("k", [1, 2, 7, 64])
def test_merge_of_oracle_runs_is_the_whole_sort(golden, name, k):
    strings = cases.CASES[name]()
    arena, offs = cases.arena_of(strings)
    rs = _cuts(len(strings), k, seed=k)
    perm, lcp = _runs_by_oracle(arena, offs, rs)
    mp, ml = pyssort.merge_runs(arena, offs, rs, perm, lcp)
    dp = hashlib.sha256(np.ascontiguousarray(mp, "<u4").tobytes()).hexdigest()
    dl = hashlib.sha256(np.ascontiguousarray(ml, "<u4").tobytes()).hexdigest()
    assert dp == golden[name]["perm_sha256"]
    assert dl == golden[name]["lcp_sha256"]


def test_merge_uint32_offsets_and_empty_runs():
    ss = pyssort.gen_urls(50_000, seed=31)
    arena, offs = ss.arena, ss.offs.astype(np.uint32)
    rs = np.array([0, 0, 10_000, 10_000, 10_001, 37_000, 50_000, 50_000], dtype=np.uint32)
    perm, lcp = _runs_by_oracle(arena, offs, rs)
    mp, ml = pyssort.merge_runs(arena, offs, rs, perm, lcp)
    rp, rl = pyoracle.oracle_sort(arena, offs)
    assert np.array_equal(mp, rp) and np.array_equal(ml, rl)


def test_merge_rejects_bad_tables():
    arena, offs = cases.arena_of([b"b", b"a", b"c"])
    perm = np.array([1, 0, 0], dtype=np.uint32)
    lcp = np.zeros(3, dtype=np.uint32)
    with pytest.raises(pyssort.SsortError):
        pyssort.merge_runs(arena, offs, np.array([0, 2], dtype=np.uint32), perm, lcp)
    with pytest.raises(pyssort.SsortError):
        pyssort.merge_runs(arena, offs, np.array([0, 2, 1, 3], dtype=np.uint32), perm, lcp)
    with pytest.raises(pyssort.SsortError):  # index 2 outside a run of 2
        pyssort.merge_runs(arena, offs, np.array([0, 2, 3], dtype=np.uint32),
                           np.array([2, 0, 0], dtype=np.uint32), lcp)


@pytest.mark.gpu
@pytest.mark.parametrize("chunk", [1, 4096, 333_333, 10**9])
def test_chunked_sort_matches_plain(sorter, chunk):
    ss = pyssort.gen_urls(1_000_000, seed=32) if chunk > 1 else pyssort.gen_urls(5000, seed=32)
    ep, el = sorter.sort_host(ss.arena, ss.offs)
    p, l = sorter.sort_host_chunked(ss.arena, ss.offs, chunk)
    assert np.array_equal(p, ep) and np.array_equal(l, el)


@pytest.mark.gpu
def test_chunked_sort_golden_duplicates(sorter, golden):
    for name in ("ut_aaa_1801", "desc_numbers_200000", "one_letter_20000"):
        arena, offs = cases.arena_of(cases.CASES[name]())
        p, l = sorter.sort_host_chunked(arena, offs, 777)
        assert hashlib.sha256(np.ascontiguousarray(p, "<u4").tobytes()).hexdigest() == \
            golden[name]["perm_sha256"], name
        assert hashlib.sha256(np.ascontiguousarray(l, "<u4").tobytes()).hexdigest() == \
            golden[name]["lcp_sha256"], name
