"""CPU tests of the synthetic workload generators (shapes and determinism)."""
import numpy as np

import pyssort


def _strings(ss, k=None):
    k = ss.n if k is None else k
    return [ss.string(i) for i in range(k)]


def test_uniform_shape_and_determinism():
    a = pyssort.gen_uniform(100000, seed=5)
    b = pyssort.gen_uniform(100000, seed=5)
    c = pyssort.gen_uniform(100000, seed=6)
    assert np.array_equal(a.arena, b.arena) and np.array_equal(a.offs, b.offs)
    assert not np.array_equal(a.arena[:1000], c.arena[:1000])
    lens = np.diff(np.append(a.offs.astype(np.int64), a.text_bytes)) - 1
    assert lens.min() == 1 and lens.max() == 20
    body = a.arena[:a.text_bytes]
    letters = body[body != 0]
    assert letters.min() == ord("a") and letters.max() == ord("z")
    assert abs(lens.mean() - 10.5) < 0.1


def test_urls_shape():
    u = pyssort.gen_urls(50000, seed=7)
    s = _strings(u, 2000)
    assert all(x.startswith(b"http://") for x in s)
    lens = np.diff(np.append(u.offs.astype(np.int64), u.text_bytes)) - 1
    assert 48 < lens.mean() < 56
    hosts = {x[7:].split(b"/")[0] for x in s}
    assert all(8 <= len(h) <= 24 for h in hosts)
    assert all(1 <= x.count(b"/") - 2 <= 6 for x in s)


def test_zipf_words_shape():
    z = pyssort.gen_zipf_words(200000, vocab=50000, seed=8)
    lens = np.diff(np.append(z.offs.astype(np.int64), z.text_bytes)) - 1
    assert lens.min() >= 1 and lens.max() <= 24
    s = _strings(z, 50000)
    distinct = len(set(s))
    assert distinct < 40000  # heavy duplication
    top = max(set(s), key=s.count)
    assert s.count(top) > 1000


def test_offsets_ascending_and_nul_terminated():
    z = pyssort.gen_uniform(1000, 0, 5, seed=9)
    assert np.all(np.diff(z.offs.astype(np.int64)) >= 1)
    ends = np.append(z.offs[1:].astype(np.int64), z.text_bytes) - 1
    assert np.all(z.arena[ends] == 0)
    assert np.all(z.arena[z.text_bytes:z.text_bytes + 16] == 0)


def test_repeat_text_shape_determinism_and_depth():
    """The suffix-sorting text: deterministic, padded with 16 zero bytes, no
    NUL inside, and its copied passages give suffix LCPs hundreds of bytes
    deep (checked with the oracle on a small text)."""
    import pyoracle
    a = pyssort.gen_repeat_text(400_000, n_repeats=20, seed=8)
    b = pyssort.gen_repeat_text(400_000, n_repeats=20, seed=8)
    c = pyssort.gen_repeat_text(400_000, n_repeats=20, seed=9)
    assert np.array_equal(a, b) and not np.array_equal(a, c)
    assert len(a) == 400_016 and not a[400_000:].any()
    assert np.count_nonzero(a[:400_000] == 0) == 0
    assert set(np.unique(a[:400_000])) <= set(range(ord("a"), ord("z") + 1)) | {ord(" ")}
    _, lcp = pyoracle.oracle_sort(a, np.arange(400_000, dtype=np.uint64))
    assert lcp.max() > 500
