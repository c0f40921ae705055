"""Text inputs: the strings of a whole file as the reference's sortstring makes
them (src/sortstring.c:310-358), found on the GPU (ssort_text_offsets_device)
and sorted (ssort_sort_text_host).  Expected string starts come from a
restatement of create_strings_delim / create_suffixes below; expected order
and LCPs from the oracle."""
import numpy as np
import pytest

import pyoracle
import pyssort


def delim_starts(text, delim):
    """create_strings_delim (src/sortstring.c:310-335): each delimiter ends a
    string, the next starts after it, the tail after the last delimiter is
    dropped; '\\n' delimiters become NUL.  Returns (starts, terminated text)."""
    buf = np.frombuffer(bytes(text), dtype=np.uint8).copy()
    ends = np.flatnonzero(buf == delim)
    starts = np.concatenate([[0], ends[:-1] + 1]).astype(np.uint64) if len(ends) else \
        np.zeros(0, dtype=np.uint64)
    if delim:
        buf[ends] = 0
    return starts, buf


def padded(buf):
    return np.concatenate([buf, np.zeros(16, dtype=np.uint8)])


def sample_text(n_lines, seed, with_tail=True):
    rng = np.random.default_rng(seed)
    words = [bytes(rng.integers(97, 123, size=int(k), dtype=np.uint8)) for k in
             rng.integers(0, 12, size=300)]
    lines = []
    for _ in range(n_lines):
        k = int(rng.integers(0, 6))
        lines.append(b" ".join(words[int(j)] for j in rng.integers(0, len(words), size=k)))
    text = b"\n".join(lines) + b"\n"
    if with_tail:
        text += b"tail without newline"
    return text


def test_delim_restatement_small_cases():
    s, buf = delim_starts(b"b\na\n\nc", ord("\n"))
    assert list(s) == [0, 2, 4]
    assert bytes(buf) == b"b\0a\0\0c"
    s, _ = delim_starts(b"abc", ord("\n"))
    assert len(s) == 0
    s, buf = delim_starts(b"x\0yy\0", 0)
    assert list(s) == [0, 2] and bytes(buf) == b"x\0yy\0"


def _expect(buf, starts):
    perm, lcp = pyoracle.oracle_sort(padded(buf), starts)
    return starts[perm], lcp


@pytest.mark.gpu
@pytest.mark.parametrize("tail", [True, False])
def test_lines_mode_matches_oracle(sorter, tail):
    text = sample_text(30_000, seed=91, with_tail=tail)
    starts, buf = delim_starts(text, ord("\n"))
    exp_offs, exp_lcp = _expect(buf, starts)
    offs, lcp = sorter.sort_text(text, pyssort.TEXT_LINES)
    assert np.array_equal(offs, exp_offs)
    assert np.array_equal(lcp, exp_lcp)


@pytest.mark.gpu
def test_raw_mode_matches_oracle(sorter):
    text = sample_text(20_000, seed=92).replace(b"\n", b"\0")
    starts, buf = delim_starts(text, 0)
    exp_offs, exp_lcp = _expect(buf, starts)
    offs, lcp = sorter.sort_text(text, pyssort.TEXT_RAW)
    assert np.array_equal(offs, exp_offs)
    assert np.array_equal(lcp, exp_lcp)


@pytest.mark.gpu
def test_suffix_mode_matches_oracle(sorter):
    """All suffixes of a text with long repeated passages (deep LCPs)."""
    rng = np.random.default_rng(93)
    parts = []
    base = sample_text(200, seed=94, with_tail=False)
    for _ in range(40):
        a = int(rng.integers(0, len(base) - 600))
        parts.append(base[a:a + int(rng.integers(50, 600))])
    text = b"".join(parts)
    buf = np.frombuffer(text, dtype=np.uint8)
    starts = np.arange(len(text), dtype=np.uint64)
    exp_offs, exp_lcp = _expect(buf, starts)
    assert exp_lcp.max() > 200  # the repeats make deep refinement necessary
    offs, lcp = sorter.sort_text(text, pyssort.TEXT_SUFFIXES)
    assert np.array_equal(offs, exp_offs)
    assert np.array_equal(lcp, exp_lcp)


@pytest.mark.gpu
@pytest.mark.parametrize("width", [4, 8])
def test_offsets_device_and_text_rewrite(sorter, width):
    torch = pytest.importorskip("torch")
    text = sample_text(50_000, seed=95) + b"\n\n\n"
    starts, buf = delim_starts(text, ord("\n"))
    d_text = torch.from_numpy(np.frombuffer(text, dtype=np.uint8).copy()).cuda()
    dt = torch.int32 if width == 4 else torch.int64
    d_offs = torch.empty(len(starts) + 5, dtype=dt, device="cuda")
    n = sorter.text_offsets_device(d_text, len(text), pyssort.TEXT_LINES, d_offs, width,
                                   len(starts) + 5)
    torch.cuda.synchronize()
    assert n == len(starts)
    got = d_offs[:n].cpu().numpy().astype(np.uint64)
    assert np.array_equal(got, starts)
    assert np.array_equal(d_text.cpu().numpy(), buf)


@pytest.mark.gpu
def test_offsets_capacity_is_checked(sorter):
    torch = pytest.importorskip("torch")
    text = b"a\nb\nc\n"
    d_text = torch.from_numpy(np.frombuffer(text, dtype=np.uint8).copy()).cuda()
    d_offs = torch.zeros(2, dtype=torch.int64, device="cuda")
    with pytest.raises(pyssort.SsortError) as e:
        sorter.text_offsets_device(d_text, len(text), pyssort.TEXT_LINES, d_offs, 8, 2)
    assert e.value.status == -1
    assert bytes(d_text.cpu().numpy()) == text  # nothing written


@pytest.mark.gpu
def test_large_lines_text_properties(sorter):
    """200 MB of lines: the oracle's independent checker on the GPU output."""
    ss = pyssort.gen_zipf_words(20_000_000, seed=96)
    buf = ss.arena[:ss.text_bytes].copy()
    buf[buf == 0] = ord("\n")
    offs, lcp = sorter.sort_text(buf, pyssort.TEXT_LINES)
    assert len(offs) == ss.n
    term = buf.copy()
    term[term == ord("\n")] = 0
    perm = np.argsort(offs, kind="stable").astype(np.uint32)  # input index of each start
    starts = np.sort(offs)
    inv = np.empty_like(perm)
    inv[perm] = np.arange(len(perm), dtype=np.uint32)
    bad, first = pyoracle.oracle_check(padded(term), starts, inv, lcp)
    assert bad == 0, first


@pytest.mark.gpu
@pytest.mark.parametrize("flags", [[], ["--raw"], ["--suffix-sorting"]])
def test_cli_sorts_checks_and_writes(tmp_path, flags):
    """ssort-sort: the file's strings, sorted, one per line (as sortstring
    --write writes them), and its --check verdict."""
    import os
    import subprocess
    cli = os.path.join(os.path.dirname(pyssort.LIB_PATH), "ssort-sort")
    text = sample_text(5_000, seed=97)
    if flags == ["--raw"]:
        text = text.replace(b"\n", b"\0")
    if flags == ["--suffix-sorting"]:
        text = text[:4000].replace(b"\n", b" ")
    src = tmp_path / "in.txt"
    src.write_bytes(text)
    out = tmp_path / "out.txt"
    r = subprocess.run([cli, *flags, "--check", "--write", str(out), str(src)],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    assert "Checking: GOOD" in r.stderr
    if flags == ["--suffix-sorting"]:
        strings = [text[i:] for i in range(len(text))]
    else:
        d = b"\0" if flags == ["--raw"] else b"\n"
        strings = text.split(d)[:-1]
    assert out.read_bytes() == b"".join(s + b"\n" for s in sorted(strings))
