"""GPU parity: the CUDA sort (through the C ABI) against the reference's own
outputs (golden fixtures from msd_CE6) and against the C oracle on seeded
workloads; full-size workloads are checked through size-independent properties
(permutation, byte order, stability, LCP) by the independent checker."""
import hashlib

import numpy as np
import pytest

import cases
import pyoracle
import pyssort

pytestmark = pytest.mark.gpu


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


@pytest.mark.parametrize("name", list(cases.CASES))
def test_golden_cases_host_api(name, golden, sorter):
    strings = cases.CASES[name]()
    arena, offs = cases.arena_of(strings)
    perm, lcp = sorter.sort_host(arena, offs)
    g = golden[name]
    if "perm" in g:
        assert perm.tolist() == g["perm"]
        assert lcp.tolist() == g["lcp"]
    assert digest(perm) == g["perm_sha256"]
    assert digest(lcp) == g["lcp_sha256"]


@pytest.mark.parametrize("name", ["ut_runs30_8001", "dup_heavy_100000", "shared8_65537",
                                  "high_bytes_5000", "desc_numbers_200000"])
def test_golden_cases_u32_offsets(name, golden, sorter):
    strings = cases.CASES[name]()
    arena, offs = cases.arena_of(strings)
    perm, lcp = sorter.sort_host(arena, offs.astype(np.uint32))
    assert digest(perm) == golden[name]["perm_sha256"]
    assert digest(lcp) == golden[name]["lcp_sha256"]


def test_unpadded_arena_tail(sorter):
    """Strings ending at the very end of the arena (no padding bytes)."""
    strings = cases.uniform(5000, 31, 0, 30)
    arena, offs = cases.arena_of(strings)
    arena = arena[: len(arena) - 16].copy()
    perm, lcp = sorter.sort_host(arena, offs)
    ref_perm, ref_lcp = pyoracle.oracle_sort(np.concatenate([arena, np.zeros(16, np.uint8)]), offs)
    assert np.array_equal(perm, ref_perm) and np.array_equal(lcp, ref_lcp)


def test_device_api_with_torch_stream(sorter):
    torch = pytest.importorskip("torch")
    strings = cases.dup_heavy(50000, 32)
    arena, offs = cases.arena_of(strings)
    d_arena = torch.from_numpy(arena).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    n = len(strings)
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    d_lcp = torch.empty(n, dtype=torch.int32, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        sorter.sort_device(d_arena, arena.nbytes, d_offs, 8, n, d_perm, d_lcp,
                           stream=s.cuda_stream)
    torch.cuda.synchronize()
    perm = d_perm.cpu().numpy().view(np.uint32)
    lcp = d_lcp.cpu().numpy().view(np.uint32)
    ref_perm, ref_lcp = pyoracle.oracle_sort(arena, offs)
    assert np.array_equal(perm, ref_perm) and np.array_equal(lcp, ref_lcp)


@pytest.mark.parametrize("name", ["ut_runs30_8001", "dup_heavy_100000", "long_prefix_10000",
                                  "all_empty_100"])
def test_permutation_without_lcp_output(name, golden, sorter):
    """A NULL lcp pointer (host and device entry points) gives the same
    permutation; the LCP is then kept in library scratch."""
    torch = pytest.importorskip("torch")
    arena, offs = cases.arena_of(cases.CASES[name]())
    perm, none = sorter.sort_host(arena, offs, with_lcp=False)
    assert none is None
    assert digest(perm) == golden[name]["perm_sha256"]
    n = len(offs)
    d_arena = torch.from_numpy(arena).cuda()
    d_offs = torch.from_numpy(offs.view(np.int64)).cuda()
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    sorter.sort_device(d_arena, arena.nbytes, d_offs, 8, n, d_perm, None)
    torch.cuda.synchronize()
    assert digest(d_perm.cpu().numpy().view(np.uint32)) == golden[name]["perm_sha256"]


def test_pointer_array_form(sorter):
    strings = cases.high_bytes(3000, 33) + cases.ut_bb_a_bbb(50)
    out, lcp = sorter.sort_strings(strings, with_lcp=True)
    order, ref_lcp = pyoracle.python_sort(strings)
    assert out == [strings[i] for i in order]
    assert lcp.tolist() == ref_lcp


@pytest.mark.parametrize("wl,n", [("uniform_1m", 1_000_000), ("urls", 2_000_000),
                                  ("zipf", 5_000_000), ("alpha4", 1_000_000),
                                  ("alpha95_long", 500_000)])
def test_workloads_against_oracle(wl, n, sorter):
    ss = {
        "uniform_1m": lambda: pyssort.gen_uniform(n, 1, 20, ord("a"), 26, 1),
        "urls": lambda: pyssort.gen_urls(n, 4096, 1.1, 2),
        "zipf": lambda: pyssort.gen_zipf_words(n, 1_000_000, 0.15, 24, 1.0, 3),
        "alpha4": lambda: pyssort.gen_uniform(n, 1, 32, ord("A"), 4, 41),
        "alpha95_long": lambda: pyssort.gen_uniform(n, 1, 128, ord(" "), 95, 42),
    }[wl]()
    perm, lcp = sorter.sort_host(ss.arena, ss.offs)
    ref_perm, ref_lcp = pyoracle.oracle_sort(ss.arena, ss.offs)
    assert np.array_equal(perm, ref_perm)
    assert np.array_equal(lcp, ref_lcp)


def test_repeatable(sorter):
    ss = pyssort.gen_urls(500_000, seed=44)
    p1, l1 = sorter.sort_host(ss.arena, ss.offs)
    p2, l2 = sorter.sort_host(ss.arena, ss.offs)
    assert np.array_equal(p1, p2) and np.array_equal(l1, l2)


@pytest.mark.parametrize("wl", ["urls_50m", "zipf_words_100m"])
def test_full_size_properties(wl, sorter):
    """The full-size plain workloads: the checker verifies permutation, byte
    order, stability and every LCP entry independently of the oracle sort."""
    ss = pyssort.WORKLOADS[wl]()
    perm, lcp = sorter.sort_host(ss.arena, ss.offs)
    bad, first = pyoracle.oracle_check(ss.arena, ss.offs, perm, lcp)
    assert bad == 0, f"{bad} violations, first at {first}"


def _tied_window_strings(n, lead, alpha, seed):
    """`lead` random bytes from the first `alpha` letters, then 8 equal bytes,
    then 6 random letters: the keys differ first in byte 0, so the 53-bit
    window after that bit ends inside the equal bytes and all strings with the
    same lead bytes tie on it."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        out.append(bytes(rng.integers(97, 97 + alpha, size=lead, dtype=np.uint8)) + b"QQQQQQQQ" +
                   bytes(rng.integers(97, 123, size=6, dtype=np.uint8)))
    return out


@pytest.mark.parametrize("prefetch,lean,merge", [(0, 0, 0), (0, 1, 0), (0, 2, 0), (1, 0, 0),
                                                (0, 0, 1)])
@pytest.mark.parametrize("n,lead,alpha,full", [(200, 2, 26, False), (1500, 2, 26, False),
                                               (700, 2, 26, False), (1500, 1, 2, True),
                                               (200, 1, 2, True), (300, 1, 2, True),
                                               (3500, 2, 26, False), (3500, 1, 2, True)])
def test_tied_packed_windows(n, lead, alpha, full, prefetch, lean, merge):
    """Segments of the one-warp (<= 256) and CTA (<= 2048) sorts whose packed
    keys tie: runs of up to 64 tied records are put in order in place, longer
    ones fall back to the full comparator; both give the oracle's order and
    LCPs, with the CTA sort single- or double-buffered and with either finish."""
    strings = _tied_window_strings(n, lead, alpha, seed=n + lead)
    arena, offs = cases.arena_of(strings)
    with pyssort.Sorter(0) as sorter:
        sorter.set_param(pyssort.SSORT_PARAM_BLOCK_PREFETCH, prefetch)
        sorter.set_param(pyssort.SSORT_PARAM_BLOCK_LEAN, lean)
        sorter.set_param(pyssort.SSORT_PARAM_WARP_MERGE, merge)
        perm, lcp = sorter.sort_host(arena, offs)
        full_sorted = sorter.stats().full_sorted
    ref_perm, ref_lcp = pyoracle.oracle_sort(arena, offs)
    assert np.array_equal(perm, ref_perm) and np.array_equal(lcp, ref_lcp)
    assert (full_sorted > 0) == full


def test_saved_round1_keys():
    """URLs (54 bytes per string): round 0's gather keeps every string's key
    bytes 16..31 and round 1 reads them instead of the arena; short strings
    (about 11 bytes each) keep none, and a sort right after a sort that sent
    few strings into round 1 keeps none either, the one after it does again.
    Results are the oracle's every time."""
    ss = pyssort.gen_urls(2_000_000, seed=48)
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    short = pyssort.gen_uniform(2_000_000, 1, 20, ord("a"), 26, 49)
    with pyssort.Sorter(0) as s:
        perm, lcp = s.sort_host(ss.arena, ss.offs)
        st = s.stats()
        assert st.window_saved == ss.n and st.window_used > 0
        assert np.array_equal(perm, rp) and np.array_equal(lcp, rl)
        s.sort_host(short.arena, short.offs)
        assert s.stats().window_saved == 0
        for saved in (0, ss.n):
            perm, lcp = s.sort_host(ss.arena, ss.offs)
            assert s.stats().window_saved == saved
            assert np.array_equal(perm, rp) and np.array_equal(lcp, rl)


def test_saved_round1_keys_batched():
    """A batched call of URL instances, small (sorted on chip in round 0) and
    large (gathered in round 0, keys kept for round 1): every instance is the
    oracle's sort of it alone."""
    sizes = [3000, 1500, 700_000, 2000, 400_000, 10, 2049, 4096, 4097]
    sets = [pyssort.gen_urls(m, seed=500 + k) for k, m in enumerate(sizes)]
    parts, offs, base = [], [], 0
    for st in sets:
        parts.append(st.arena[:st.text_bytes])
        offs.append(st.offs + np.uint64(base))
        base += st.text_bytes
    arena = np.concatenate(parts + [np.zeros(16, np.uint8)])
    offs = np.concatenate(offs)
    inst = np.zeros(len(sizes) + 1, dtype=np.uint32)
    inst[1:] = np.cumsum(sizes)
    with pyssort.Sorter(0) as s:
        p, l = s.sort_batch_host(arena, offs, inst)
        st = s.stats()
    assert st.window_saved == sum(m for m in sizes if m > 2048) and st.window_used > 0
    for k in range(len(sizes)):
        lo, hi = int(inst[k]), int(inst[k + 1])
        rp, rl = pyoracle.oracle_sort(arena, offs[lo:hi])
        assert np.array_equal(p[lo:hi], rp), k
        assert np.array_equal(l[lo:hi], rl), k


def test_saved_round1_keys_u32_offsets():
    """Kept round-1 keys with 4-byte offsets (the width whole-text sorts use)."""
    ss = pyssort.gen_urls(1_500_000, seed=51)
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    with pyssort.Sorter(0) as s:
        p, l = s.sort_host(ss.arena, ss.offs.astype(np.uint32))
        assert s.stats().window_saved == ss.n
    assert np.array_equal(p, rp) and np.array_equal(l, rl)


def test_pointer_array_one_large_span(sorter):
    """The drop-in's fast path: every pointer inside one readable span of
    more than 128 MB (copied through the pinned staging chunks), sorted
    pointers rebuilt from the sorted offsets; the order is the oracle's."""
    import ctypes
    ss = pyssort.gen_urls(3_000_000, seed=71)
    assert ss.text_bytes > (128 << 20)
    base = ss.arena.ctypes.data
    ptrs = (ctypes.c_void_p * ss.n)(*[base + int(o) for o in ss.offs])
    lcp = np.empty(ss.n, dtype=np.uint32)
    rc = pyssort.lib().ssort_sort_strings(sorter._ctx, ptrs, ss.n, lcp.ctypes.data)
    assert rc == 0, pyssort.lib().ssort_last_error()
    got = np.array([p - base for p in ptrs], dtype=np.uint64)
    perm = np.searchsorted(ss.offs, got).astype(np.uint32)  # offsets ascend with the index
    ref_perm, ref_lcp = pyoracle.oracle_sort(ss.arena, ss.offs)
    assert np.array_equal(perm, ref_perm)
    assert np.array_equal(lcp, ref_lcp)


@pytest.mark.parametrize("n", [2047, 2048, 2049, 3000, 4096, 8192])
def test_cta_sort_cutoff(n, sorter):
    """Inputs at and above the CTA sort's 2048-string cutoff: up to 2048
    strings are sorted on chip without a partition pass, larger inputs are
    partitioned first (round 0: the whole input; round 1: the shared-prefix
    case's single segment).  Both match the oracle."""
    for strings in (cases.uniform(n, 900 + n), cases.shared8(n, 950 + n)):
        arena, offs = cases.arena_of(strings)
        perm, lcp = sorter.sort_host(arena, offs)
        st = sorter.stats()
        ref_perm, ref_lcp = pyoracle.oracle_sort(arena, offs)
        assert np.array_equal(perm, ref_perm) and np.array_equal(lcp, ref_lcp)
        assert (st.partitioned == 0) == (n <= 2048)
