"""CPU tests of the oracle: pinned against the reference's own outputs (golden
fixtures made by running msd_CE6) and, when oracle/_ref is built, against the
reference library directly; plus the checker's ability to catch planted
mistakes (planted in oracle output, on the CPU)."""
import hashlib

import numpy as np
import pytest

import cases
import pyoracle


def digest(a):
    return hashlib.sha256(np.ascontiguousarray(a, dtype="<u4").tobytes()).hexdigest()


@pytest.mark.parametrize("name", list(cases.CASES))
def test_oracle_matches_golden(name, golden):
    strings = cases.CASES[name]()
    arena, offs = cases.arena_of(strings)
    perm, lcp = pyoracle.oracle_sort(arena, offs)
    g = golden[name]
    assert g["n"] == len(strings)
    assert digest(perm) == g["perm_sha256"]
    assert digest(lcp) == g["lcp_sha256"]
    if "perm" in g:
        assert perm.tolist() == g["perm"]
        assert lcp.tolist() == g["lcp"]


@pytest.mark.parametrize("name", [n for n in cases.CASES if not n.startswith(("desc", "shared8_655"))])
def test_python_definition_matches_golden(name, golden):
    """The golden permutation is the stable sort by bytes (definition check)."""
    strings = cases.CASES[name]()
    if len(strings) > 120000:
        pytest.skip("large")
    order, lcp = pyoracle.python_sort(strings)
    assert digest(np.array(order, dtype=np.uint32)) == golden[name]["perm_sha256"]
    assert digest(np.array(lcp, dtype=np.uint32)) == golden[name]["lcp_sha256"]


def test_reference_unit_test_expectations():
    """The content checks of the reference's test_routines
    (unit-test/main.cpp:228-248) and insertion-sort KATs (:172-204)."""
    strings = cases.CASES["kat_insertion5"]()
    arena, offs = cases.arena_of(strings)
    perm, _ = pyoracle.oracle_sort(arena, offs)
    assert [strings[i] for i in perm] == [b"", b"aaaaa", b"bbaaa", b"bbbbb", b"c"]
    strings = cases.CASES["kat_insertion_depth"]()
    arena, offs = cases.arena_of(strings)
    perm, _ = pyoracle.oracle_sort(arena, offs)
    assert [strings[i] for i in perm] == [b"aaaa2", b"aaaa3", b"bbbb1"]
    for k in range(1, 1000, 200):
        strings = cases.ut_bb_a_bbb(k)
        arena, offs = cases.arena_of(strings)
        perm, _ = pyoracle.oracle_sort(arena, offs)
        out = [strings[i] for i in perm]
        assert out == [b"a"] * k + [b"bb"] * k + [b"bbb"] * k


@pytest.mark.skipif(not pyoracle.have_ref(), reason="oracle/_ref not built")
@pytest.mark.parametrize("gen", ["uniform", "urls", "zipf", "alpha4"])
def test_oracle_matches_reference_library(gen):
    import pyssort
    ss = {
        "uniform": lambda: pyssort.gen_uniform(300000, seed=21),
        "urls": lambda: pyssort.gen_urls(200000, seed=22),
        "zipf": lambda: pyssort.gen_zipf_words(300000, vocab=30000, seed=23),
        "alpha4": lambda: pyssort.gen_uniform(200000, 1, 32, ord("A"), 4, seed=24),
    }[gen]()
    perm, lcp = pyoracle.oracle_sort(ss.arena, ss.offs)
    p6 = pyoracle.ref_sort_perm("msd_CE6", ss.arena, ss.offs)
    assert np.array_equal(perm, p6)
    bad, _ = pyoracle.oracle_check(ss.arena, ss.offs, perm, lcp)
    assert bad == 0


def test_checker_catches_planted_mistakes():
    strings = cases.dup_heavy(5000, 99)
    arena, offs = cases.arena_of(strings)
    perm, lcp = pyoracle.oracle_sort(arena, offs)
    assert pyoracle.oracle_check(arena, offs, perm, lcp)[0] == 0
    # order violation
    p = perm.copy()
    i = next(k for k in range(1, len(p)) if strings[p[k - 1]] != strings[p[k]])
    p[i - 1], p[i] = p[i], p[i - 1]
    assert pyoracle.oracle_check(arena, offs, p, None)[0] > 0
    # stability violation: swap two equal strings
    p = perm.copy()
    j = next(k for k in range(1, len(p)) if strings[p[k - 1]] == strings[p[k]])
    p[j - 1], p[j] = p[j], p[j - 1]
    assert pyoracle.oracle_check(arena, offs, p, None)[0] > 0
    # not a permutation
    p = perm.copy()
    p[3] = p[4]
    assert pyoracle.oracle_check(arena, offs, p, None)[0] > 0
    # wrong lcp
    l = lcp.copy()
    l[len(l) // 2] += 1
    assert pyoracle.oracle_check(arena, offs, perm, l)[0] > 0


def test_oracle_pointer_form_sorts_in_place():
    import ctypes
    strings = [b"pear", b"apple", b"", b"apple", b"\xffz", b"ap"]
    bufs = [ctypes.create_string_buffer(s) for s in strings]
    arr = (ctypes.c_void_p * len(bufs))(*[ctypes.addressof(b) for b in bufs])
    pyoracle.oracle().oracle_msd(arr, len(bufs))
    got = [ctypes.string_at(arr[i]) for i in range(len(bufs))]
    assert got == sorted(strings)
    # stability: the two "apple" keep input order
    first_apple = [i for i in range(len(bufs)) if got[i] == b"apple"][0]
    assert arr[first_apple] == ctypes.addressof(bufs[1])
