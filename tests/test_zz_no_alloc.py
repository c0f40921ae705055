"""GPU test of ssort_sort_device_noalloc, the entry point for callers that
cannot let the library allocate device memory (its scratch is a fixed array
inside the library).  It must return exactly what ssort_sort_device returns for
the same input, and what the oracle returns, call after call, although every
call reuses the same scratch.

Kept in its own file named to be collected last, so a failure here cannot hide
the rest of the suite; it also passes when run alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

import pyoracle
import pyssort

pytestmark = pytest.mark.gpu

MAX_N = 262144  # SSORT_NOALLOC_MAX_N in include/ssort_b200.h


def _device_set(ss, off_dtype):
    torch = pytest.importorskip("torch")
    arena = torch.from_numpy(np.ascontiguousarray(ss.arena)).cuda()
    offs_np = ss.offs.astype(off_dtype)
    offs = torch.from_numpy(offs_np.view(np.int64 if off_dtype == np.uint64 else np.int32)).cuda()
    return arena, offs, offs_np.dtype.itemsize


def _sort_noalloc(arena, nbytes, offs, width, n, with_lcp=True, stream=None):
    torch = pytest.importorskip("torch")
    perm = torch.empty(max(n, 1), dtype=torch.int32, device="cuda")
    lcp = torch.empty(max(n, 1), dtype=torch.int32, device="cuda") if with_lcp else None
    st = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
    rc = pyssort.lib().ssort_sort_device_noalloc(arena.data_ptr(), nbytes, offs.data_ptr(), width,
                                                 n, perm.data_ptr(),
                                                 lcp.data_ptr() if with_lcp else None, st)
    assert rc == 0, pyssort.lib().ssort_last_error().decode()
    p = perm.cpu().numpy().view(np.uint32)[:n]
    return p, (lcp.cpu().numpy().view(np.uint32)[:n] if with_lcp else None)


def _sort_regular(sorter, arena, nbytes, offs, width, n):
    torch = pytest.importorskip("torch")
    perm = torch.empty(n, dtype=torch.int32, device="cuda")
    lcp = torch.empty(n, dtype=torch.int32, device="cuda")
    sorter.sort_device(arena, nbytes, offs, width, n, perm, lcp)
    torch.cuda.synchronize()
    return perm.cpu().numpy().view(np.uint32), lcp.cpu().numpy().view(np.uint32)


def test_noalloc_matches_regular_entry_point_twice():
    with pyssort.Sorter(0) as sorter:
        sets = [
            (pyssort.gen_urls(MAX_N, seed=61), np.uint64),          # deep prefixes, partitions
            (pyssort.gen_zipf_words(200_000, vocab=5000, seed=62), np.uint32),  # duplicates
            (pyssort.gen_uniform(3000, 0, 30, 1, 255, seed=63), np.uint64),     # small, high bytes
        ]
        for ss, od in sets:
            arena, offs, width = _device_set(ss, od)
            ref_perm, ref_lcp = _sort_regular(sorter, arena, ss.arena.nbytes, offs, width, ss.n)
            for _ in range(2):  # two calls in a row on the shared scratch
                perm, lcp = _sort_noalloc(arena, ss.arena.nbytes, offs, width, ss.n)
                assert np.array_equal(perm, ref_perm)
                assert np.array_equal(lcp, ref_lcp)


def test_noalloc_matches_oracle_on_caller_stream_and_without_lcp():
    torch = pytest.importorskip("torch")
    ss = pyssort.gen_urls(100_000, seed=64)
    ref_perm, ref_lcp = pyoracle.oracle_sort(ss.arena, ss.offs)
    arena, offs, width = _device_set(ss, np.uint64)
    side = torch.cuda.Stream()
    for _ in range(2):
        perm, lcp = _sort_noalloc(arena, ss.arena.nbytes, offs, width, ss.n, stream=side)
        assert np.array_equal(perm, ref_perm)
        assert np.array_equal(lcp, ref_lcp)
        perm, none = _sort_noalloc(arena, ss.arena.nbytes, offs, width, ss.n, with_lcp=False)
        assert none is None
        assert np.array_equal(perm, ref_perm)


@pytest.mark.parametrize("n", [1, 2])
def test_noalloc_tiny_inputs(n):
    ss = pyssort.gen_uniform(n, 0, 5, ord("a"), 3, seed=65 + n)
    ref_perm, ref_lcp = pyoracle.oracle_sort(ss.arena, ss.offs)
    arena, offs, width = _device_set(ss, np.uint32)
    for _ in range(2):
        perm, lcp = _sort_noalloc(arena, ss.arena.nbytes, offs, width, n)
        assert np.array_equal(perm, ref_perm)
        assert np.array_equal(lcp, ref_lcp)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    L = pyssort.lib()
    rc = L.ssort_sort_device_noalloc(ctypes.c_void_p(16), 64, ctypes.c_void_p(16), 8, MAX_N + 1,
                                     ctypes.c_void_p(16), None, None)
    assert rc == -1
    assert b"exceeds the fixed scratch" in L.ssort_last_error()
