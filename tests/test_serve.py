"""GPU tests of the request server (ssort_server_*): continuous batching must
not change any result.  Every request is checked against the same request
sorted alone through the plain entry point, and small ones against the
oracle, whatever it shared the rounds with."""
import hashlib

import numpy as np
import pytest

import cases
import pyoracle
import pyssort

pytestmark = pytest.mark.gpu


def _requests(ninst, seed, hi, off_dtypes=(np.uint32, np.uint64)):
    params = pyssort.batch_instance_params(ninst, seed=seed, lo=2, hi=hi)
    ss = pyssort.gen_instances(params, seed=seed + 1)
    reqs = []
    for i in range(len(params)):
        arena, offs = ss.request(i, off_dtypes[i % len(off_dtypes)])
        reqs.append((arena.copy(), offs))
    return reqs


def _alone(sorter, reqs):
    return [sorter.sort_host(a, o) for a, o in reqs]


def _check(results, expected):
    for k, ((perm, lcp), (ep, el)) in enumerate(zip(results, expected)):
        assert np.array_equal(perm, ep), f"request {k}: perm differs from the sort alone"
        assert np.array_equal(lcp, el), f"request {k}: lcp differs from the sort alone"


def test_serve_all_at_once_matches_alone_and_oracle(sorter):
    reqs = _requests(40, seed=81, hi=300_000)
    expected = _alone(sorter, reqs)
    with pyssort.Server(64 << 20, 4_000_000) as srv:
        subs = [srv.submit(a, o) for a, o in reqs]
        done = srv.drain()
        assert sorted(done) == sorted(s[0] for s in subs)
        info = srv.info()
        assert info["max_active"] > 1
        assert info["arena_in_use"] == 0 and info["strings_in_use"] == 0
    _check([(p, l) for _, p, l in subs], expected)
    for (a, o), (_, p, l) in zip(reqs, subs):
        if len(o) <= 20_000:
            rp, rl = pyoracle.oracle_sort(a, o.astype(np.uint64))
            assert np.array_equal(p, rp) and np.array_equal(l, rl)


def test_serve_requests_join_mid_flight(sorter):
    """Later requests join while earlier ones are several rounds deep."""
    first = _requests(4, seed=82, hi=3_000_000)
    later = _requests(30, seed=84, hi=100_000)
    expected = _alone(sorter, first + later)
    with pyssort.Server(512 << 20, 16_000_000) as srv:
        subs = [srv.submit(a, o) for a, o in first]
        done = []
        for _ in range(2):
            done += srv.step()
        assert srv.info()["rounds"] >= 1
        for a, o in later:
            subs.append(srv.submit(a, o))
            done += srv.step()
        done += srv.drain()
        assert sorted(done) == sorted(s[0] for s in subs)
        assert all(srv.poll(s[0]) == pyssort.REQ_DONE for s in subs)
        assert srv.info()["max_active"] >= 2
    _check([(p, l) for _, p, l in subs], expected)


def test_serve_budget_admits_one_request_at_a_time(sorter):
    reqs = []
    for k in range(12):
        ss = pyssort.gen_uniform(50_000 + 1000 * k, 1, 20, ord("a"), 26, seed=860 + k)
        reqs.append((ss.arena[:ss.text_bytes].copy(), ss.offs.copy()))
    sizes = [(a.nbytes + 1 + 255) // 256 * 256 for a, _ in reqs]
    budget = max(sizes)
    assert 2 * min(sizes) > budget  # no two requests fit the pool together
    expected = _alone(sorter, reqs)
    with pyssort.Server(budget, 400_000) as srv:
        subs = [srv.submit(a, o) for a, o in reqs]
        states = [srv.poll(s[0]) for s in subs]
        assert all(st == pyssort.REQ_QUEUED for st in states)
        srv.drain()
        info = srv.info()
        assert info["max_active"] == 1
        assert info["requests_done"] == len(reqs)
    _check([(p, l) for _, p, l in subs], expected)


def test_serve_golden_cases_and_edges(sorter, golden):
    names = [n for n in cases.CASES if len(cases.CASES[n]()) < 70000]
    with pyssort.Server(64 << 20, 1_000_000) as srv:
        subs = {}
        for k, name in enumerate(names):
            arena, offs = cases.arena_of(cases.CASES[name]())
            dt = np.uint32 if k % 2 else np.uint64
            subs[name] = srv.submit(arena, offs.astype(dt))
        srv.drain()
    for name, (_, perm, lcp) in subs.items():
        dp = hashlib.sha256(np.ascontiguousarray(perm, "<u4").tobytes()).hexdigest()
        dl = hashlib.sha256(np.ascontiguousarray(lcp, "<u4").tobytes()).hexdigest()
        assert dp == golden[name]["perm_sha256"], name
        assert dl == golden[name]["lcp_sha256"], name


def test_serve_ragged_arena_edges(sorter):
    """Offsets at or past the request's arena end and an unterminated last
    string read as the single-request sort reads them: NUL past the end."""
    arena = np.frombuffer(b"banana\0apple\0cherry", dtype=np.uint8).copy()
    offs = np.array([0, 7, 13, 19, 40, 2, 16], dtype=np.uint64)
    other = np.frombuffer(b"zzzzzzzzzzzzzzzzzzzzzzzzzzzzzzzz\0", dtype=np.uint8).copy()
    ooffs = np.arange(0, 30, 3, dtype=np.uint32)
    ep, el = sorter.sort_host(arena, offs)
    op, ol = sorter.sort_host(other, ooffs)
    with pyssort.Server(1 << 20, 10_000) as srv:
        _, p2, l2 = srv.submit(other, ooffs)
        _, p1, l1 = srv.submit(arena, offs)
        _, pe, le = srv.submit(np.zeros(0, np.uint8), np.zeros(0, np.uint64))
        _, ps, ls = srv.submit(arena, np.array([3], dtype=np.uint32))
        srv.drain()
    assert np.array_equal(p1, ep) and np.array_equal(l1, el)
    assert np.array_equal(p2, op) and np.array_equal(l2, ol)
    assert len(pe) == 0
    assert list(ps) == [0] and list(ls) == [0]


def test_serve_rejects_bad_requests():
    with pyssort.Server(4096, 1000) as srv:
        a, o = cases.arena_of([b"x" * 5000])
        with pytest.raises(pyssort.SsortError) as e:
            srv.submit(a, o)
        assert e.value.status == -2
        a, o = cases.arena_of([b"y"] * 1001)
        with pytest.raises(pyssort.SsortError) as e:
            srv.submit(a, o)
        assert e.value.status == -2
        with pytest.raises(pyssort.SsortError) as e:
            srv.poll(12345)
        assert e.value.status == -1
        # the server still works after rejected requests
        a, o = cases.arena_of([b"b", b"a"])
        rid, perm, lcp = srv.submit(a, o)
        srv.drain()
        assert list(perm) == [1, 0] and list(lcp) == [0, 0]


def test_serve_device_resident_requests(sorter):
    """Requests whose buffers are in device memory (copied device to device)
    mixed with host requests give the same results."""
    torch = pytest.importorskip("torch")
    reqs = _requests(16, seed=88, hi=400_000, off_dtypes=(np.uint32,))
    expected = _alone(sorter, reqs)
    dev = []
    with pyssort.Server(256 << 20, 8_000_000) as srv:
        subs = []
        for k, (a, o) in enumerate(reqs):
            if k % 2:
                subs.append(("host",) + srv.submit(a, o)[1:])
                continue
            d_a = torch.from_numpy(a).cuda()
            d_o = torch.from_numpy(o.view(np.int32)).cuda()
            d_p = torch.empty(len(o), dtype=torch.int32, device="cuda")
            d_l = torch.empty(len(o), dtype=torch.int32, device="cuda")
            srv.submit_ptr(d_a, a.nbytes, d_o, 4, len(o), d_p, d_l)
            dev.append((d_a, d_o))
            subs.append(("dev", d_p, d_l))
        srv.drain()
    got = []
    for kind, p, l in subs:
        if kind == "dev":
            p = p.cpu().numpy().view(np.uint32)
            l = l.cpu().numpy().view(np.uint32)
        got.append((p, l))
    _check(got, expected)
