"""Tuning parameters and the autotuner: every parameter value gives the same
perm and LCP (checked against the default and the oracle), out-of-range
values are rejected, and ssort_autotune picks values from its candidate sets,
records them, and later sorts of the same class stay bit-exact."""
import hashlib

import numpy as np
import pytest

import cases
import pyoracle
import pyssort

pytestmark = pytest.mark.gpu

SETTINGS = [
    (pyssort.SSORT_PARAM_WARP8_CAP, 64),
    (pyssort.SSORT_PARAM_WARP8_CAP, 128),
    (pyssort.SSORT_PARAM_OVERLAP, 0),
    (pyssort.SSORT_PARAM_FUSED_GATHER, 0),
    (pyssort.SSORT_PARAM_FUSED_GATHER, 2),
    (pyssort.SSORT_PARAM_TARGET_BUCKET, 128),
    (pyssort.SSORT_PARAM_TARGET_BUCKET, 1024),
    (pyssort.SSORT_PARAM_WARP1_DEEP, 0),
    (pyssort.SSORT_PARAM_WARP1_DEEP, 1),
    (pyssort.SSORT_PARAM_WARP1_DEEP, 4096),
    (pyssort.SSORT_PARAM_BLOCK_PREFETCH, 0),
    (pyssort.SSORT_PARAM_BLOCK_PREFETCH, 1),
    (pyssort.SSORT_PARAM_L2_PREFETCH, 1),
    (pyssort.SSORT_PARAM_GRAPH, 1),
    (pyssort.SSORT_PARAM_DIGIT_BITS, 8),
    (pyssort.SSORT_PARAM_DIGIT_BITS, 9),
    (pyssort.SSORT_PARAM_SCATTER, 1),
    (pyssort.SSORT_PARAM_SCATTER, 2),
    (pyssort.SSORT_PARAM_BLOCK_LEAN, 1),
    (pyssort.SSORT_PARAM_BLOCK_LEAN, 2),
    (pyssort.SSORT_PARAM_GRAPH, 2),
    (pyssort.SSORT_PARAM_MATCH_VOTE, 1),
    (pyssort.SSORT_PARAM_WARP_MERGE, 0),
    (pyssort.SSORT_PARAM_SCAN, 0),
]


@pytest.mark.parametrize("param,value", SETTINGS)
def test_parameter_values_keep_results(golden, param, value):
    with pyssort.Sorter(0) as s:
        s.set_param(param, value)
        for name in ("desc_numbers_200000", "long_prefix_10000", "high_bytes_5000",
                     "ut_runs30_8001", "one_letter_20000"):
            arena, offs = cases.arena_of(cases.CASES[name]())
            p, l = s.sort_host(arena, offs)
            assert hashlib.sha256(np.ascontiguousarray(p, "<u4").tobytes()).hexdigest() == \
                golden[name]["perm_sha256"], name
            assert hashlib.sha256(np.ascontiguousarray(l, "<u4").tobytes()).hexdigest() == \
                golden[name]["lcp_sha256"], name
        ss = pyssort.gen_urls(300_000, seed=61)
        p, l = s.sort_host(ss.arena, ss.offs)
        rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
        assert np.array_equal(p, rp) and np.array_equal(l, rl)


@pytest.mark.parametrize("deep", [0, 1, 2, 64, 4096])
def test_in_warp_refinement_on_deep_suffixes(deep):
    """Suffixes of a text with copied passages: runs of two or three strings
    sharing hundreds of bytes, refined in the warp (up to `deep` 16-byte steps
    per round, the rest in later rounds); results are the oracle's under every
    step limit, including limits that leave runs for the next round."""
    text = pyssort.gen_repeat_text(300_000, n_repeats=40, seed=12)
    offs = np.arange(300_000, dtype=np.uint64)
    rp, rl = pyoracle.oracle_sort(text, offs)
    assert rl.max() > 500
    with pyssort.Sorter(0) as s:
        s.set_param(pyssort.SSORT_PARAM_WARP1_DEEP, deep)
        p, l = s.sort_host(text, offs)
        st = s.stats()
    assert np.array_equal(p, rp) and np.array_equal(l, rl)
    if deep == 0:
        assert st.warp1_deep == 0
    else:
        assert st.warp1_deep > 0
    if deep >= 64:
        assert st.rounds < 20  # without the refinement: about max lcp / 16 rounds


def test_out_of_range_parameters_are_rejected():
    with pyssort.Sorter(0) as s:
        for param, value in [(pyssort.SSORT_PARAM_WARP8_CAP, 32),
                             (pyssort.SSORT_PARAM_WARP8_CAP, 512),
                             (pyssort.SSORT_PARAM_OVERLAP, 2),
                             (pyssort.SSORT_PARAM_FUSED_GATHER, -1),
                             (pyssort.SSORT_PARAM_FUSED_GATHER, 3),
                             (pyssort.SSORT_PARAM_TARGET_BUCKET, 4096),
                             (pyssort.SSORT_PARAM_WARP1_DEEP, -1),
                             (pyssort.SSORT_PARAM_WARP1_DEEP, 4097),
                             (pyssort.SSORT_PARAM_BLOCK_PREFETCH, 2),
                             (pyssort.SSORT_PARAM_L2_PREFETCH, 2),
                             (pyssort.SSORT_PARAM_GRAPH, 3),
                             (pyssort.SSORT_PARAM_BLOCK_LEAN, 3),
                             (pyssort.SSORT_PARAM_MATCH_VOTE, 2),
                             (pyssort.SSORT_PARAM_WARP_MERGE, 2),
                             (pyssort.SSORT_PARAM_SCAN, 2),
                             (pyssort.SSORT_PARAM_GRAPH_MAX_LEVELS, 0),
                             (pyssort.SSORT_PARAM_DIGIT_BITS, 7),
                             (pyssort.SSORT_PARAM_DIGIT_BITS, 11),
                             (pyssort.SSORT_PARAM_SCATTER, 3),
                             (99, 1)]:
            with pytest.raises(pyssort.SsortError) as e:
                s.set_param(param, value)
            assert e.value.status == -1


def test_autotune_then_sort_stays_exact():
    torch = pytest.importorskip("torch")
    ss = pyssort.gen_urls(1_000_000, seed=62)
    d_arena = torch.from_numpy(ss.arena).cuda()
    d_offs = torch.from_numpy(ss.offs.view(np.int64)).cuda()
    with pyssort.Sorter(0) as s:
        t = s.autotune(d_arena, ss.arena.nbytes, d_offs, 8, ss.n)
        assert t["size_class"] == 19  # floor(log2(1e6))
        assert t["entropy_class"] in (0, 1, 2)
        assert 0 < t["entropy_bits"] <= 8
        assert t["target_bucket"] in (256, 512, 1024)
        assert t["warp8_cap"] in (64, 128, 256)
        assert t["overlap"] in (0, 1) and t["fused_gather"] in (0, 1)
        assert t["tuned_ms"] <= t["default_ms"]
        assert t["digit_bits"] in (8, 9, 10)
        assert t["block_prefetch"] in (0, 1) and t["l2_prefetch"] in (0, 1)
        assert t["graph"] in (0, 1)
        # base, then every other candidate of every knob
        assert t["trials"] == 2 + 2 * (2 + 2 + 2 + 1 + 1 + 1 + 1 + 2 + 1)
        # a later sort of the same class uses the recorded values
        d_perm = torch.empty(ss.n, dtype=torch.int32, device="cuda")
        d_lcp = torch.empty(ss.n, dtype=torch.int32, device="cuda")
        s.sort_device(d_arena, ss.arena.nbytes, d_offs, 8, ss.n, d_perm, d_lcp)
        torch.cuda.synchronize()
        rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
        assert np.array_equal(d_perm.cpu().numpy().view(np.uint32), rp)
        assert np.array_equal(d_lcp.cpu().numpy().view(np.uint32), rl)


def test_kept_keys_with_separate_gather():
    """With the fused gather off, round 1's separate gather reads the key
    copies round 0 kept (2 M URLs: above the size where copies are kept)."""
    ss = pyssort.gen_urls(2_000_000, seed=63)
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    with pyssort.Sorter(0) as s:
        s.set_param(pyssort.SSORT_PARAM_FUSED_GATHER, 0)
        p, l = s.sort_host(ss.arena, ss.offs)
        st = s.stats()
    assert st.gather_fused == 0 and st.window_saved > 0 and st.window_used > 0
    assert np.array_equal(p, rp) and np.array_equal(l, rl)


@pytest.mark.parametrize("mode,graph", [(1, 0), (1, 1), (2, 0), (2, 1)])
def test_round0_gather_inside_count(mode, graph):
    """Round 0's first partition level gathers its keys inside the count and
    keeps key bytes 16..31 there for round 1, under mode 2 and, for a round 0
    of at most 4 M keys (here 2 M URLs), under the default mode 1; in the host
    loop and in the device-driven loop."""
    ss = pyssort.gen_urls(2_000_000, seed=64)
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    with pyssort.Sorter(0) as s:
        s.set_param(pyssort.SSORT_PARAM_FUSED_GATHER, mode)
        s.set_param(pyssort.SSORT_PARAM_GRAPH, graph)
        p, l = s.sort_host(ss.arena, ss.offs)
        st = s.stats()
    assert st.gather_fused == st.gather_elems > 0
    assert st.window_saved > 0 and st.window_used > 0
    assert np.array_equal(p, rp) and np.array_equal(l, rl)


def test_batched_sort_uses_per_class_tuning():
    """After autotuning plain sorts of two size classes, a batched call
    partitions each segment with the bucket size tuned for its own size
    class; every instance is still the oracle's result."""
    torch = pytest.importorskip("torch")
    with pyssort.Sorter(0) as s:
        for n in (300_000, 40_000):
            ss = pyssort.gen_uniform(n, 1, 20, ord("a"), 26, seed=n)
            d_arena = torch.from_numpy(ss.arena).cuda()
            d_offs = torch.from_numpy(ss.offs.view(np.int64)).cuda()
            s.autotune(d_arena, ss.arena.nbytes, d_offs, 8, ss.n)
        params = pyssort.batch_instance_params(120, 41, lo=2, hi=400_000)
        b = pyssort.gen_instances(params, seed=42)
        perm, lcp = s.sort_batch_host(b.arena, b.offs, b.inst_start)
    st = b.inst_start
    for i in range(len(params)):
        lo, hi = int(st[i]), int(st[i + 1])
        if hi - lo < 1:
            continue
        rp, rl = pyoracle.oracle_sort(b.arena, b.offs[lo:hi])
        assert np.array_equal(perm[lo:hi], rp), i
        assert np.array_equal(lcp[lo:hi], rl), i
