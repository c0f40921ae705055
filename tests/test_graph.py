"""The device-driven round loop (SSORT_PARAM_GRAPH): the sort runs as a CUDA
graph whose rounds and partition levels are conditional loops driven by the
device's own counters.  It must give the oracle's (and the host loop's) perm
and LCP on every input, match the host loop's statistics, relaunch itself
when a sort needs more rounds than one launch runs, reuse its graph across
calls on the same buffers, and turn an exhausted level budget into an error
status that leaves the context usable."""
import hashlib

import numpy as np
import pytest

import cases
import pyoracle
import pyssort

pytestmark = pytest.mark.gpu


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


def graph_sorter():
    s = pyssort.Sorter(0)
    s.set_param(pyssort.SSORT_PARAM_GRAPH, 1)
    return s


@pytest.mark.parametrize("name", ["desc_numbers_200000", "long_prefix_10000", "high_bytes_5000",
                                  "ut_runs30_8001", "one_letter_20000", "all_empty_100",
                                  "equal_long_70000", "shared8_65537"])
def test_graph_golden_cases(golden, name):
    if name not in cases.CASES:
        pytest.skip("no such case")
    arena, offs = cases.arena_of(cases.CASES[name]())
    with graph_sorter() as s:
        p, l = s.sort_host(arena, offs)
    assert digest(p) == golden[name]["perm_sha256"]
    assert digest(l) == golden[name]["lcp_sha256"]


@pytest.mark.parametrize("wl,n", [("urls_50m", 2_000_000), ("zipf_words_100m", 2_000_000),
                                  ("uniform_1m", 1_000_000)])
def test_graph_matches_oracle_and_host_loop(wl, n):
    ss = pyssort.WORKLOADS[wl](n / {"urls_50m": 50e6, "zipf_words_100m": 100e6,
                                    "uniform_1m": 1e6}[wl])
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    with pyssort.Sorter(0) as h:
        hp, hl = h.sort_host(ss.arena, ss.offs)
        hst = h.stats()
    with graph_sorter() as s:
        for _ in range(2):  # the second call reuses the graph
            p, l = s.sort_host(ss.arena, ss.offs)
            assert np.array_equal(p, rp) and np.array_equal(l, rl)
        st = s.stats()
    assert np.array_equal(hp, rp) and np.array_equal(hl, rl)
    # same work in both loops
    assert st.rounds == hst.rounds
    assert st.partition_levels == hst.partition_levels
    assert st.partitioned == hst.partitioned
    assert list(st.live)[:st.rounds] == list(hst.live)[:hst.rounds]


def test_graph_batched_instances():
    params = pyssort.batch_instance_params(300, 21, lo=2, hi=200_000)
    ss = pyssort.gen_instances(params, seed=22)
    with graph_sorter() as s:
        perm, lcp = s.sort_batch_host(ss.arena, ss.offs, ss.inst_start)
    st = ss.inst_start
    for i in range(len(params)):
        lo, hi = int(st[i]), int(st[i + 1])
        if hi - lo < 1:
            continue
        rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs[lo:hi])
        assert np.array_equal(perm[lo:hi], rp), i
        assert np.array_equal(lcp[lo:hi], rl), i


def test_graph_relaunches_past_its_round_budget():
    """Long shared prefixes with in-warp refinement off: 100+ rounds, more
    than one graph launch runs (64), so the host relaunches the graph."""
    rng = np.random.default_rng(5)
    prefix = bytes(rng.integers(97, 123, size=1800, dtype=np.uint8))
    strings = [prefix + bytes(rng.integers(97, 100, size=6, dtype=np.uint8)) for _ in range(3000)]
    arena, offs = cases.arena_of(strings)
    rp, rl = pyoracle.oracle_sort(arena, offs)
    with graph_sorter() as s:
        s.set_param(pyssort.SSORT_PARAM_WARP1_DEEP, 0)
        p, l = s.sort_host(arena, offs)
        st = s.stats()
    assert st.rounds > 64
    assert np.array_equal(p, rp) and np.array_equal(l, rl)


def test_graph_level_budget_is_an_error_not_a_hang():
    """A round that needs a second partition level under a budget of one
    level stops with SSORT_EINTERNAL; the context then sorts normally."""
    ss = pyssort.gen_urls(2_000_000, seed=23)
    with graph_sorter() as s:
        s.set_param(pyssort.SSORT_PARAM_GRAPH_MAX_LEVELS, 1)
        with pytest.raises(pyssort.SsortError) as e:
            s.sort_host(ss.arena, ss.offs)
        assert e.value.status == -5
        assert b"partition levels exceeded" in pyssort.lib().ssort_last_error()
        s.set_param(pyssort.SSORT_PARAM_GRAPH_MAX_LEVELS, 4096)
        p, l = s.sort_host(ss.arena, ss.offs)
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    assert np.array_equal(p, rp) and np.array_equal(l, rl)


def test_graph_rebuilds_for_new_buffers():
    with graph_sorter() as s:
        for seed in (31, 32, 33):
            ss = pyssort.gen_uniform(50_000 + seed, 0, 24, ord("a"), 4, seed=seed)
            p, l = s.sort_host(ss.arena, ss.offs)
            rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
            assert np.array_equal(p, rp) and np.array_equal(l, rl)


def test_auto_mode_uses_the_graph_from_the_second_identical_sort():
    """SSORT_PARAM_GRAPH = 2: a sort whose buffers and size differ from the
    previous sort's runs on the host loop; the second sort in a row with the
    same arguments builds and runs the graph, and so do later ones; results
    stay the oracle's throughout."""
    torch = pytest.importorskip("torch")
    ss = pyssort.gen_urls(400_000, seed=24)
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    d_arena = torch.from_numpy(ss.arena).cuda()
    d_offs = torch.from_numpy(ss.offs.view(np.int64)).cuda()
    d_perm = torch.empty(ss.n, dtype=torch.int32, device="cuda")
    d_lcp = torch.empty(ss.n, dtype=torch.int32, device="cuda")
    used = []
    with pyssort.Sorter(0) as s:
        s.set_param(pyssort.SSORT_PARAM_GRAPH, 2)
        for _ in range(3):
            s.sort_device(d_arena, ss.arena.nbytes, d_offs, 8, ss.n, d_perm, d_lcp)
            torch.cuda.synchronize()
            used.append(s.stats().graph_launches)
            assert np.array_equal(d_perm.cpu().numpy().view(np.uint32), rp)
            assert np.array_equal(d_lcp.cpu().numpy().view(np.uint32), rl)
    assert used[0] == 0 and used[1] >= 1 and used[2] >= 1


def test_graph_with_single_pass_scan():
    """The device-driven loop with the decoupled look-back scan inside its
    level loop (its state cleared by a memset node each level)."""
    ss = pyssort.gen_zipf_words(2_000_000, vocab=20_000, seed=25)
    rp, rl = pyoracle.oracle_sort(ss.arena, ss.offs)
    with graph_sorter() as s:
        s.set_param(pyssort.SSORT_PARAM_SCAN, 1)
        for _ in range(2):
            p, l = s.sort_host(ss.arena, ss.offs)
            assert np.array_equal(p, rp) and np.array_equal(l, rl)
