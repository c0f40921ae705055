"""Randomised parity sweep: many seeded string sets of different shapes
(alphabet size, length distribution, shared prefixes, duplicate runs, sizes
around the segment-class cutoffs) sorted on the GPU through the host entry
point and the batched entry point, each compared with the oracle (perm and
LCP, bit-exact).  Plus inputs that need hundreds of 16-byte rounds."""
import numpy as np
import pytest

import pyoracle
import pyssort

pytestmark = pytest.mark.gpu


def _make(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.choice([1, 2, 7, 33, 257, 513, 1025, 2049, 5000, 30000, 120000]))
    alpha = int(rng.choice([1, 2, 4, 26, 95, 255]))
    lo = int(rng.choice([1, 32, 97, 200])) if alpha < 255 else 1
    lo = min(lo, 256 - alpha)
    prefix = bytes(rng.integers(lo, lo + alpha, size=int(rng.choice([0, 0, 5, 17, 40, 130])),
                                dtype=np.uint8))
    kind = rng.integers(3)
    if kind == 0:
        lens = rng.integers(0, int(rng.choice([4, 20, 70])) + 1, size=n)
    elif kind == 1:
        lens = np.minimum(rng.geometric(0.2, size=n) - 1, 60)
    else:
        lens = np.full(n, int(rng.integers(0, 40)))
    strings = []
    for L in lens:
        strings.append(prefix + bytes(rng.integers(lo, lo + alpha, size=int(L), dtype=np.uint8)))
    # duplicate runs: copy some strings over others
    if rng.random() < 0.5 and n > 4:
        for _ in range(int(rng.integers(1, 6))):
            src = int(rng.integers(n))
            cnt = int(rng.integers(1, max(2, n // 3)))
            for d in rng.integers(0, n, size=cnt):
                strings[int(d)] = strings[src]
    return strings


def _arena(strings):
    offs = np.zeros(len(strings), dtype=np.uint64)
    if strings:
        offs[1:] = np.cumsum([len(s) + 1 for s in strings])[:-1]
    arena = np.frombuffer(b"".join(s + b"\0" for s in strings) + b"\0" * 16, dtype=np.uint8)
    return arena.copy(), offs


@pytest.mark.parametrize("seed", range(40))
def test_random_sets_match_oracle(sorter, seed):
    strings = _make(1000 + seed)
    arena, offs = _arena(strings)
    rp, rl = pyoracle.oracle_sort(arena, offs)
    p, l = sorter.sort_host(arena, offs.astype(np.uint32) if seed % 2 else offs)
    assert np.array_equal(p, rp)
    assert np.array_equal(l, rl)


def test_random_sets_as_one_batch(sorter):
    sets = [_make(2000 + k) for k in range(24)]
    strings = [s for st in sets for s in st]
    arena, offs = _arena(strings)
    inst = np.zeros(len(sets) + 1, dtype=np.uint32)
    inst[1:] = np.cumsum([len(st) for st in sets])
    p, l = sorter.sort_batch_host(arena, offs, inst)
    for k in range(len(sets)):
        lo, hi = int(inst[k]), int(inst[k + 1])
        if hi == lo:
            continue
        rp, rl = pyoracle.oracle_sort(arena, offs[lo:hi])
        assert np.array_equal(p[lo:hi], rp), k
        assert np.array_equal(l[lo:hi], rl), k


def test_hundreds_of_rounds(sorter):
    """3000 strings sharing a 4000-byte prefix (250 rounds of 16 bytes), with
    duplicates, and 2000 copies of one 1500-byte string."""
    rng = np.random.default_rng(77)
    pre = bytes(rng.integers(97, 100, size=4000, dtype=np.uint8))
    tails = [bytes(rng.integers(97, 100, size=int(k), dtype=np.uint8))
             for k in rng.integers(0, 30, size=1500)]
    strings = [pre + tails[int(i)] for i in rng.integers(0, len(tails), size=3000)]
    strings += [b"z" * 1500] * 2000
    strings += [pre[:int(k)] for k in rng.integers(0, 4000, size=500)]
    perm_in = rng.permutation(len(strings))
    strings = [strings[int(i)] for i in perm_in]
    arena, offs = _arena(strings)
    rp, rl = pyoracle.oracle_sort(arena, offs)
    p, l = sorter.sort_host(arena, offs)
    assert np.array_equal(p, rp)
    assert np.array_equal(l, rl)
    assert int(l.max()) >= 4000
    assert sorter.stats().rounds > 200


def _deep_families(seed):
    """Small groups whose runs need many 16-byte steps, each family behind
    its own first byte; the last string is an unterminated copy of the one
    before it, running to the end of the arena."""
    rng = np.random.default_rng(seed)

    def rand(n, a=2):
        return bytes(rng.integers(97, 97 + a, size=n, dtype=np.uint8))
    s = [b"A" + b"x" * 5000] * 32                      # one run of 32
    for _ in range(3):                                   # identical pairs past 8 KB
        t = b"B" + rand(20000)
        s += [t, t]
    for _ in range(4):                                   # differ in the last byte
        t = b"C" + rand(3000)
        s += [t + b"a", t + b"b"]
    for _ in range(4):                                   # one a prefix of the other
        t = b"D" + rand(2500)
        s += [t, t + rand(int(rng.integers(1, 40)))]
    for k in range(3, 9):                                # runs of 3..8 sharing 700 bytes
        t = b"E" + bytes([96 + k]) + rand(700)
        s += [t + rand(int(rng.integers(0, 300))) for _ in range(k)]
    order = rng.permutation(len(s))
    s = [s[int(i)] for i in order]
    last = b"F" + rand(3000)
    return s + [last, last]


@pytest.mark.parametrize("deep", [1, 3, 64, 4096])
def test_in_warp_refinement_edges(deep):
    strings = _deep_families(90)
    body = b"".join(x + b"\0" for x in strings[:-1]) + strings[-1]  # last one unterminated
    arena = np.frombuffer(body, dtype=np.uint8).copy()
    offs = np.zeros(len(strings), dtype=np.uint64)
    offs[1:] = np.cumsum([len(x) + 1 for x in strings])[:-1]
    rp, rl = pyoracle.oracle_sort(np.concatenate([arena, np.zeros(16, np.uint8)]), offs)
    assert int(rl.max()) >= 20000
    with pyssort.Sorter(0) as s:
        s.set_param(pyssort.SSORT_PARAM_WARP1_DEEP, deep)
        p, l = s.sort_host(arena, offs)
        assert s.stats().warp1_deep > 0
    assert np.array_equal(p, rp)
    assert np.array_equal(l, rl)
