"""CPU tests of the C ABI: the library loads, exports every entry point the
public header declares, and validates arguments without touching a GPU."""
import ctypes
import os
import re

import pytest

import pyssort

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ssort_b200.h")


def header_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    text = re.sub(r"//[^\n]*", "", text)
    names = re.findall(r"^[A-Za-z_][\w\s\*]*?\b(\w+)\s*\([^;{]*\)\s*;", text, flags=re.M)
    return sorted(set(names))


def test_header_parses():
    fns = header_functions()
    assert "msd_gpu" in fns and "ssort_sort_device" in fns
    assert set(fns) == set(pyssort.EXPORTS)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(pyssort.LIB_PATH)
    for name in header_functions():
        assert hasattr(lib, name), name


def test_routine_signature_symbol():
    """msd_gpu has the struct routine::f signature: void(unsigned char**, size_t)."""
    lib = pyssort.lib()
    fn = lib.msd_gpu
    assert fn.restype is None
    assert len(fn.argtypes) == 2


def test_status_strings():
    L = pyssort.lib()
    assert L.ssort_strerror(0) == b"ok"
    assert L.ssort_strerror(-1) == b"invalid argument"
    assert L.ssort_strerror(-4) == b"no CUDA device"


def test_no_device_is_reported_not_faked():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pyssort.SsortError) as e:
        pyssort.Sorter(0)
    assert e.value.status == -4


def test_null_context_is_rejected():
    L = pyssort.lib()
    assert L.ssort_sort_host(None, None, 0, None, 8, 0, None, None) == -1
    assert L.ssort_sort_device(None, None, 0, None, 8, 0, None, None, None) == -1
    assert L.ssort_set_profiling(None, 1) == -1


def test_server_without_device_is_reported():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(pyssort.SsortError) as e:
        pyssort.Server(1 << 20, 1000)
    assert e.value.status == -4


def test_null_server_is_rejected():
    import ctypes
    L = pyssort.lib()
    rid = ctypes.c_uint64()
    st = ctypes.c_int()
    assert L.ssort_server_submit(None, None, 0, None, 8, 0, None, None, ctypes.byref(rid)) == -1
    assert L.ssort_server_step(None, None, 0, None) == -1
    assert L.ssort_server_poll(None, 1, ctypes.byref(st)) == -1
    assert L.ssort_server_drain(None) == -1
    L.ssort_server_destroy(None)
    out = ctypes.c_void_p()
    assert L.ssort_server_create(0, 1 << 20, 0, ctypes.byref(out)) == -1


@pytest.mark.parametrize("cname,pyname", [("ssort_stats", "Stats"),
                                          ("ssort_server_info", "ServerInfo"),
                                          ("ssort_tuning", "Tuning")])
def test_ctypes_structs_match_header_layout(tmp_path, cname, pyname):
    """The ctypes mirrors of the header's result structs: same size and the
    same offset for every field, as the C compiler lays them out."""
    import shutil
    import subprocess
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no C compiler")
    cls = getattr(pyssort, pyname)
    fields = [f for f, _ in cls._fields_]
    src = tmp_path / "layout.c"
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "ssort_b200.h"',
             "int main(void) {", f'    printf("%zu\\n", sizeof({cname}));']
    lines += [f'    printf("%zu\\n", offsetof({cname}, {f}));' for f in fields]
    lines += ["    return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run([cc, "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True,
                                          text=True).stdout.split()]
    assert got[0] == ctypes.sizeof(cls)
    assert got[1:] == [getattr(cls, f).offset for f in fields]
