"""The drop-in boundary: the reference's own drivers, compiled from its sources
with msd_gpu registered through ROUTINE_REGISTER, run unchanged on the GPU.

  oracle/_ref/unit-test    reference unit-test/main.cpp: runs every registered
                           routine, msd_gpu included, on its three families
  oracle/_ref/sortstring   reference CLI: `sortstring --check msd_gpu <file>`
"""
import os
import subprocess

import numpy as np
import pytest

import pyssort

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF = os.path.join(ROOT, "oracle", "_ref")
UNIT = os.path.join(REF, "unit-test")
CLI = os.path.join(REF, "sortstring")

pytestmark = pytest.mark.gpu


@pytest.mark.skipif(not os.path.exists(UNIT), reason="oracle/_ref/unit-test not built")
def test_reference_unit_test_runs_msd_gpu():
    r = subprocess.run([UNIT], stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "[msd_gpu]" in r.stdout
    assert "*** All OK ***" in r.stdout


@pytest.mark.skipif(not os.path.exists(CLI), reason="oracle/_ref/sortstring not built")
@pytest.mark.parametrize("raw", [False, True])
def test_sortstring_cli_check(tmp_path, raw):
    ss = pyssort.gen_urls(300_000, seed=51)
    body = bytes(ss.arena[: ss.text_bytes])
    if not raw:
        body = body.replace(b"\0", b"\n")
    f = tmp_path / "input.txt"
    f.write_bytes(body)
    out = tmp_path / "out.txt"
    args = [CLI, "--check", f"--write={out}"] + (["--raw"] if raw else []) + ["msd_gpu", str(f)]
    r = subprocess.run(args, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stdout[-3000:]
    assert "Check: GOOD" in r.stdout
    lines = out.read_bytes().split(b"\n")[:-1]
    strings = [ss.string(i) for i in range(ss.n)]
    assert lines == sorted(strings)


def test_msd_gpu_symbol_sorts_separately_allocated_strings():
    """msd_gpu called through its C signature on strdup-like separate buffers
    (the unit test's layout, unit-test/main.cpp:220-270)."""
    import ctypes
    rng = np.random.default_rng(52)
    strings = [bytes(rng.integers(1, 256, size=int(rng.integers(0, 30)), dtype=np.uint8))
               for _ in range(20000)]
    bufs = [ctypes.create_string_buffer(s) for s in strings]
    arr = (ctypes.c_void_p * len(bufs))(*[ctypes.addressof(b) for b in bufs])
    pyssort.lib().msd_gpu(arr, len(bufs))
    pos = {ctypes.addressof(b): i for i, b in enumerate(bufs)}
    order = [pos[arr[i]] for i in range(len(bufs))]
    assert order == sorted(range(len(strings)), key=lambda i: (strings[i], i))
