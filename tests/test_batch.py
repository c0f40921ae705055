"""GPU parity of the batched entry points: every instance of a batch must come
out exactly as if it had been sorted alone (perm local to the instance, lcp
restarting at 0), checked against the oracle instance by instance."""
import numpy as np
import pytest

import cases
import pyoracle
import pyssort

pytestmark = pytest.mark.gpu


def _check_instances(ss, perm, lcp):
    inst = ss.inst_start
    for i in range(len(inst) - 1):
        lo, hi = int(inst[i]), int(inst[i + 1])
        if hi == lo:
            continue
        ref_perm, ref_lcp = pyoracle.oracle_sort(ss.arena, ss.offs[lo:hi])
        assert np.array_equal(perm[lo:hi], ref_perm), f"instance {i}"
        assert np.array_equal(lcp[lo:hi], ref_lcp), f"instance {i}"


def test_batch_mixed_instances_host_api(sorter):
    params = [(c, L, lo, sz) for (c, L, (lo, sz)) in [
        (5000, 8, pyssort.BATCH_ALPHABETS[0]), (1, 32, pyssort.BATCH_ALPHABETS[1]),
        (70000, 128, pyssort.BATCH_ALPHABETS[2]), (2, 8, pyssort.BATCH_ALPHABETS[0]),
        (300, 32, pyssort.BATCH_ALPHABETS[1]), (33, 8, pyssort.BATCH_ALPHABETS[0]),
        (2049, 8, pyssort.BATCH_ALPHABETS[0]), (120000, 8, pyssort.BATCH_ALPHABETS[0]),
    ]]
    ss = pyssort.gen_instances(params, seed=71)
    perm, lcp = sorter.sort_batch_host(ss.arena, ss.offs, ss.inst_start)
    _check_instances(ss, perm, lcp)


def test_batch_device_api_matches_single_sorts(sorter):
    torch = pytest.importorskip("torch")
    params = pyssort.batch_instance_params(40, seed=72, hi=200_000)
    ss = pyssort.gen_instances(params, seed=73)
    d_arena = torch.from_numpy(ss.arena).cuda()
    d_offs = torch.from_numpy(ss.offs.view(np.int64)).cuda()
    d_inst = torch.from_numpy(ss.inst_start.view(np.int32)).cuda()
    n = ss.n
    d_perm = torch.empty(n, dtype=torch.int32, device="cuda")
    d_lcp = torch.empty(n, dtype=torch.int32, device="cuda")
    sorter.sort_batch_device(d_arena, ss.arena.nbytes, d_offs, 8, n, d_inst,
                             len(ss.inst_start) - 1, d_perm, d_lcp)
    torch.cuda.synchronize()
    perm = d_perm.cpu().numpy().view(np.uint32)
    lcp = d_lcp.cpu().numpy().view(np.uint32)
    # each instance alone through the plain entry point
    for i in range(len(ss.inst_start) - 1):
        lo, hi = int(ss.inst_start[i]), int(ss.inst_start[i + 1])
        p1, l1 = sorter.sort_host(ss.arena, ss.offs[lo:hi])
        assert np.array_equal(perm[lo:hi], p1) and np.array_equal(lcp[lo:hi], l1)


def test_batch_of_golden_cases(sorter, golden):
    """All golden recipes as one batch: each must reproduce the reference."""
    import hashlib
    names = [n for n in cases.CASES if len(cases.CASES[n]()) < 70000]
    sets = [cases.CASES[n]() for n in names]
    strings = [s for st in sets for s in st]
    arena, offs = cases.arena_of(strings)
    inst = np.zeros(len(sets) + 1, dtype=np.uint32)
    inst[1:] = np.cumsum([len(st) for st in sets])
    perm, lcp = sorter.sort_batch_host(arena, offs, inst)
    for i, name in enumerate(names):
        lo, hi = int(inst[i]), int(inst[i + 1])
        dp = hashlib.sha256(np.ascontiguousarray(perm[lo:hi], "<u4").tobytes()).hexdigest()
        dl = hashlib.sha256(np.ascontiguousarray(lcp[lo:hi], "<u4").tobytes()).hexdigest()
        assert dp == golden[name]["perm_sha256"], name
        assert dl == golden[name]["lcp_sha256"], name


def test_batch_rejects_bad_instance_table(sorter):
    ss = pyssort.gen_uniform(100, seed=74)
    with pytest.raises(pyssort.SsortError):
        sorter.sort_batch_host(ss.arena, ss.offs, np.array([0, 50, 40, 100], dtype=np.uint32))
    with pytest.raises(pyssort.SsortError):
        sorter.sort_batch_host(ss.arena, ss.offs, np.array([0, 99], dtype=np.uint32))
