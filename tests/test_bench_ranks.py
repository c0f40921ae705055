"""The multi-rank plumbing of bench.py on the CPU: two gloo ranks, each with
its own time; the reported time is the max over ranks and the rate is the
whole job's (replicas: every rank sorts its own copy)."""
import os
import socket

import pytest

import bench


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        mine = [0.25, 0.75][rank]
        out[rank] = bench.max_over_ranks(dist, mine, "cpu")
    finally:
        dist.destroy_process_group()


def test_max_over_two_gloo_ranks():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert out[0] == out[1] == 0.75


def test_single_process_and_job_rate():
    assert bench.max_over_ranks(None, 1.5, "cpu") == 1.5
    # two replicas of 50M strings, 10 steps, slowest rank 2 s
    assert bench.job_rate(50_000_000, 10, 2, 2.0) == pytest.approx(5e8)


@pytest.mark.parametrize("workload", ["batch_c4", "serve_c5"])
def test_reference_arm_times_instances_alone(workload):
    """The CPU reference arm of the batched and served workloads sorts a
    bounded prefix of their instance list, instance by instance."""
    ss = bench.instance_sample(workload, 20_000)
    assert len(ss.inst_start) >= 2 and ss.n == int(ss.inst_start[-1])
    t, kind = bench.time_cpu_instances(ss)
    assert t > 0 and kind in ("reference", "port")


def test_intrinsic_live_counts_strings_per_8_byte_round():
    """Strings live at depth 8r: those sharing >= 8r bytes with a neighbour
    (the definition, counted directly)."""
    import numpy as np
    rng = np.random.default_rng(3)
    for _ in range(20):
        n = int(rng.integers(1, 500))
        lcp = rng.integers(0, int(rng.integers(1, 200)), size=n).astype(np.uint32)
        lcp[0] = 0
        nb = np.maximum(lcp, np.append(lcp[1:], 0)).astype(np.int64)
        want = [n] + [int((nb >= d).sum()) for d in range(8, int(nb.max()) + 1, 8)]
        assert bench.intrinsic_live(lcp, n) == want
    assert bench.intrinsic_live(np.zeros(0, np.uint32), 0) == [0]


def test_text_workload_cpu_sample():
    """The CPU timer of the suffix workload reads the first m suffixes of the
    text (uint64 offsets 0..m-1 into it)."""
    import numpy as np
    text, tlen, mode, host_mode, host_text, n, starts_of = bench.text_workload(
        "suffixes_160m", 0.001)
    assert tlen == 160_000 and n == tlen and len(text) == tlen + 16
    assert np.array_equal(host_text(), text[:tlen])
    ss = bench.TextSample(text, starts_of, n).first(5000)
    assert ss.offs.dtype == np.uint64 and list(ss.offs[:3]) == [0, 1, 2]
    t, kind = bench.time_cpu_sort(ss, 5000)
    assert t > 0 and kind in ("reference", "port")


def test_kernel_bytes_with_kept_windows():
    """Algorithmic bytes of the gathering kernels: round 0's gather reads and
    writes 16 more bytes per kept window; a key read from a kept copy skips
    the offset (W bytes), in whichever kernel gathers round 1's first level."""
    from types import SimpleNamespace as NS
    base = dict(gather_elems=150, gather_fused=50, partitioned=300, warp1_fresh=0,
                warp1_keyed=0, warp8_fresh=0, warp8_keyed=0, block_fresh=0, block_keyed=0,
                equal_moved=0, equal_final=0)
    w = 8
    plain = bench.kernel_bytes(NS(**base, window_saved=0, window_used=0), w)
    assert plain["gather"] == 100 * (4 + w + 32)
    assert plain["count_gather"] == 50 * (4 + w + 32)
    kept = bench.kernel_bytes(NS(**base, window_saved=100, window_used=40), w)
    assert kept["gather"] == plain["gather"] + 100 * 32
    assert kept["count_gather"] == plain["count_gather"] - 40 * w
    base["gather_fused"] = 0  # separate gather in every round: it reads the copies
    sep = bench.kernel_bytes(NS(**base, window_saved=100, window_used=40), w)
    assert sep["gather"] == 150 * (4 + w + 32) + 100 * 32 - 40 * w
    assert sep["count_gather"] == 0
    base["gather_fused"] = 150  # round 0 gathers inside its count too
    fused = bench.kernel_bytes(NS(**base, window_saved=100, window_used=40), w)
    assert fused["gather"] == 0
    assert fused["count_gather"] == 150 * (4 + w + 32) + 100 * 32 - 40 * w
