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
