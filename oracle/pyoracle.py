"""TEST INFRASTRUCTURE ONLY: ctypes binding of the oracle libraries.

  liboracle.so      the C restatement of the reference's msd_CE6 (msd_oracle.c)
  _ref/libref.so    the reference's own routines compiled from its sources

Imported only by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
leg, always as the checker or the timed CPU baseline, never as the sort being
measured or shipped.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_PATH = os.path.join(HERE, "liboracle.so")
REF_PATH = os.path.join(HERE, "_ref", "libref.so")

_o = None
_r = None


def oracle():
    global _o
    if _o is None:
        L = ctypes.CDLL(ORACLE_PATH)
        vp = ctypes.c_void_p
        L.oracle_sort_arena.argtypes = [vp, vp, ctypes.c_int, ctypes.c_size_t, vp, vp]
        L.oracle_sort_ptrs.argtypes = [vp, ctypes.c_size_t, vp, vp]
        L.oracle_check_arena.argtypes = [vp, vp, ctypes.c_int, ctypes.c_size_t, vp, vp,
                                         ctypes.POINTER(ctypes.c_size_t)]
        L.oracle_check_arena.restype = ctypes.c_size_t
        L.oracle_msd.argtypes = [vp, ctypes.c_size_t]
        L.oracle_msd.restype = None
        _o = L
    return _o


def have_ref():
    return os.path.exists(REF_PATH)


def ref():
    global _r
    if _r is None:
        L = ctypes.CDLL(REF_PATH)
        vp = ctypes.c_void_p
        L.ref_sort.argtypes = [ctypes.c_char_p, vp, ctypes.c_size_t]
        L.ref_sort_arena_perm.argtypes = [ctypes.c_char_p, vp, vp, ctypes.c_size_t, vp]
        L.ref_is_multicore.argtypes = [ctypes.c_char_p]
        _r = L
    return _r


def oracle_sort(arena, offs):
    """(perm, lcp) of the stable byte-order sort, by the C restatement."""
    arena = np.ascontiguousarray(arena, dtype=np.uint8)
    offs = np.ascontiguousarray(offs)
    n = offs.shape[0]
    perm = np.empty(n, dtype=np.uint32)
    lcp = np.empty(n, dtype=np.uint32)
    rc = oracle().oracle_sort_arena(arena.ctypes.data, offs.ctypes.data, offs.dtype.itemsize, n,
                                    perm.ctypes.data, lcp.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"oracle failed ({rc})")
    return perm, lcp


def oracle_check(arena, offs, perm, lcp=None):
    """Independent validity check: (violations, first bad position)."""
    arena = np.ascontiguousarray(arena, dtype=np.uint8)
    offs = np.ascontiguousarray(offs)
    fb = ctypes.c_size_t()
    bad = oracle().oracle_check_arena(arena.ctypes.data, offs.ctypes.data, offs.dtype.itemsize,
                                      offs.shape[0], perm.ctypes.data,
                                      None if lcp is None else lcp.ctypes.data, ctypes.byref(fb))
    return int(bad), int(fb.value)


def ref_sort_perm(name, arena, offs):
    """Run the reference routine `name` over the arena; returns the index
    permutation it produced (offsets must be distinct and ascending)."""
    arena = np.ascontiguousarray(arena, dtype=np.uint8)
    offs = np.ascontiguousarray(offs, dtype=np.uint64)
    n = offs.shape[0]
    perm = np.empty(n, dtype=np.uint32)
    rc = ref().ref_sort_arena_perm(name.encode(), arena.ctypes.data, offs.ctypes.data, n,
                                   perm.ctypes.data)
    if rc != 0:
        raise RuntimeError(f"reference routine {name} failed ({rc})")
    return perm


def python_sort(strings):
    """Pure-Python definition for tiny cases: stable sort by bytes, and the
    lcp array of the sorted order."""
    order = sorted(range(len(strings)), key=lambda i: (strings[i], i))
    lcp = [0] * len(strings)
    for k in range(1, len(order)):
        a, b = strings[order[k - 1]], strings[order[k]]
        l = 0
        while l < len(a) and l < len(b) and a[l] == b[l]:
            l += 1
        lcp[k] = l
    return order, lcp


def arena_from_strings(strings):
    """Pack a list of bytes objects (no NULs) into (arena, uint64 offsets)."""
    offs = np.zeros(len(strings), dtype=np.uint64)
    parts = []
    pos = 0
    for i, s in enumerate(strings):
        offs[i] = pos
        parts.append(s + b"\0")
        pos += len(s) + 1
    arena = np.frombuffer(b"".join(parts) + b"\0" * 16, dtype=np.uint8).copy()
    return arena, offs
