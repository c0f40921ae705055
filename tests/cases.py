"""Deterministic string-set recipes shared by the golden-fixture generator
(tests/golden/make_golden.py) and the parity tests.

The first group restates the inputs of the reference's own unit test
(rantala/string-sorting unit-test/main.cpp): the insertion-sort known-answer
inputs (:172-204) and the three routine families (:220-270).  The rest are the
edge cases the sort must get bit-exact: empty input, empty strings, bytes
0x80-0xFF and 0xFF runs, long shared prefixes, descending zero-padded numbers
(the input that trips msd_CE7/CE8's sortedness shortcut), sizes on both sides
of every internal cutoff (32, 2048 strings per segment, 65536 for the
reference's superalphabet switch), and duplicate-heavy sets.
"""
import numpy as np


def _rng(seed):
    return np.random.default_rng(seed)


def _rand_strings(rng, n, lo, hi, alpha_lo, alpha_size):
    lens = rng.integers(lo, hi + 1, size=n)
    flat = rng.integers(alpha_lo, alpha_lo + alpha_size, size=int(lens.sum()), dtype=np.uint8)
    out, pos = [], 0
    for L in lens:
        out.append(flat[pos:pos + L].tobytes())
        pos += L
    return out


def ut_aaa(k):
    return [b"aaa"] * k


def ut_bb_a_bbb(k):
    return [b"bb", b"a", b"bbb"] * k


def ut_runs30(k):
    return [bytes([ord("a") + (i % 30)]) * 9 for i in range(k)]


def high_bytes(n, seed):
    return _rand_strings(_rng(seed), n, 0, 40, 1, 255)


def ff_runs(n, seed):
    rng = _rng(seed)
    return [b"\xff" * int(L) + (b"\xfe" if rng.integers(2) else b"") for L in rng.integers(0, 21, n)]


def desc_numbers(n):
    return [b"%08d" % (n - i) for i in range(n)]


def long_prefix(n, seed, plen=100):
    rng = _rng(seed)
    pre = b"p" * plen
    tails = _rand_strings(rng, n // 2, 0, 6, ord("a"), 3)
    return [pre + tails[int(i)] for i in rng.integers(0, len(tails), n)]


def one_letter(n, seed, maxlen=300):
    rng = _rng(seed)
    return [b"a" * int(L) for L in rng.integers(0, maxlen + 1, n)]


def shared8(n, seed):
    """n strings sharing the 8-byte prefix 'prefix__' (so round 1 sees one
    segment of exactly n strings)."""
    rng = _rng(seed)
    return [b"prefix__" + t for t in _rand_strings(rng, n, 0, 12, ord("a"), 4)]


def uniform(n, seed, lo=1, hi=20, alpha_lo=ord("a"), alpha_size=26):
    return _rand_strings(_rng(seed), n, lo, hi, alpha_lo, alpha_size)


def dup_heavy(n, seed, vocab=500):
    rng = _rng(seed)
    words = _rand_strings(rng, vocab, 1, 24, ord("a"), 26)
    ranks = np.minimum(rng.zipf(1.3, size=n), vocab) - 1
    return [words[int(r)] for r in ranks]


def equal_long(n, L=40):
    return [b"x" * L] * n


# name -> zero-argument builder.  Sizes keep the whole golden file small and
# the oracle well under a second per case.
CASES = {}
for _k in range(1, 2000, 200):
    CASES[f"ut_aaa_{_k}"] = (lambda k=_k: ut_aaa(k))
for _k in range(1, 1000, 200):
    CASES[f"ut_bb_a_bbb_{_k}"] = (lambda k=_k: ut_bb_a_bbb(k))
for _k in range(1, 10000, 2000):
    CASES[f"ut_runs30_{_k}"] = (lambda k=_k: ut_runs30(k))
CASES.update({
    "kat_insertion5": lambda: [b"c", b"", b"bbaaa", b"aaaaa", b"bbbbb"],
    "kat_insertion_depth": lambda: [b"bbbb1", b"aaaa3", b"aaaa2"],
    "empty_set": lambda: [],
    "single": lambda: [b"x"],
    "single_empty": lambda: [b""],
    "two_equal": lambda: [b"ab", b"ab"],
    "all_empty_100": lambda: [b""] * 100,
    "high_bytes_5000": lambda: high_bytes(5000, 11),
    "ff_runs_3000": lambda: ff_runs(3000, 12),
    "desc_numbers_200000": lambda: desc_numbers(200000),
    "long_prefix_10000": lambda: long_prefix(10000, 13),
    "one_letter_20000": lambda: one_letter(20000, 14),
    "uniform_100000": lambda: uniform(100000, 15),
    "uniform_alpha4_50000": lambda: uniform(50000, 16, 1, 32, ord("A"), 4),
    "uniform_alpha95_50000": lambda: uniform(50000, 17, 1, 128, ord(" "), 95),
    "dup_heavy_100000": lambda: dup_heavy(100000, 18),
    "equal_long_70000": lambda: equal_long(70000),
})
for _n in (31, 32, 33, 2047, 2048, 2049, 4097, 65535, 65536, 65537):
    CASES[f"shared8_{_n}"] = (lambda n=_n: shared8(n, 100 + n))


def arena_of(strings):
    """(arena uint8 with 16 zero bytes of padding, uint64 offsets)."""
    offs = np.zeros(len(strings), dtype=np.uint64)
    lens = np.fromiter((len(s) + 1 for s in strings), dtype=np.uint64, count=len(strings))
    if len(strings):
        offs[1:] = np.cumsum(lens)[:-1]
    arena = np.frombuffer(b"".join(s + b"\0" for s in strings) + b"\0" * 16, dtype=np.uint8)
    return arena.copy(), offs


def lcp_of(strings, perm):
    """LCP array of strings in perm order, by the reference's lcp() definition
    (src/mergesort_lcp.cpp:88-100), lcp[0] = 0."""
    out = np.zeros(len(perm), dtype=np.uint32)
    for k in range(1, len(perm)):
        a, b = strings[perm[k - 1]], strings[perm[k]]
        m = min(len(a), len(b))
        l = 0
        while l < m and a[l] == b[l]:
            l += 1
        out[k] = l
    return out
