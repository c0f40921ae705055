"""ctypes binding of libssort_b200.so (the C ABI in include/ssort_b200.h) and of
the synthetic workload generators in libssort_workloads.so.

This is the Python face of the product path used by the tests and the
benchmark.  It never falls back to a CPU implementation: if the CUDA library is
missing or no GPU is present, every sort raises.
"""
import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libssort_b200.so")
WLIB_PATH = os.path.join(_HERE, "libssort_workloads.so")

SSORT_OK = 0
SSORT_MAX_ROUNDS = 64

# Every symbol include/ssort_b200.h declares.
EXPORTS = (
    "msd_gpu", "ssort_strerror", "ssort_last_error", "ssort_ctx_create", "ssort_ctx_destroy",
    "ssort_sort_device", "ssort_sort_host", "ssort_sort_strings", "ssort_get_stats",
    "ssort_set_profiling", "ssort_get_kernel_times", "ssort_sort_device_noalloc",
    "ssort_set_param", "ssort_sort_batch_device", "ssort_sort_batch_host",
    "ssort_server_create", "ssort_server_destroy", "ssort_server_submit", "ssort_server_step",
    "ssort_server_poll", "ssort_server_drain", "ssort_server_get_info",
    "ssort_text_offsets_device", "ssort_sort_text_host", "ssort_pinned_alloc",
    "ssort_pinned_free", "ssort_merge_runs", "ssort_sort_host_chunked", "ssort_autotune",
)
# text input modes (sortstring's default line mode, --raw, --suffix-sorting)
TEXT_LINES, TEXT_RAW, TEXT_SUFFIXES = 0, 1, 2
# request states reported by ssort_server_poll
REQ_QUEUED, REQ_LOADING, REQ_ACTIVE, REQ_DRAINING, REQ_DONE = range(5)
SSORT_PARAM_TARGET_BUCKET = 1
SSORT_PARAM_WARP8_CAP = 2
SSORT_PARAM_OVERLAP = 3
SSORT_PARAM_FUSED_GATHER = 4
SSORT_PARAM_WARP1_DEEP = 5
SSORT_PARAM_BLOCK_PREFETCH = 6
SSORT_PARAM_GRAPH = 7
SSORT_PARAM_GRAPH_MAX_LEVELS = 8
SSORT_PARAM_L2_PREFETCH = 9
SSORT_PARAM_DIGIT_BITS = 10
SSORT_PARAM_SCATTER = 11
SSORT_PARAM_BLOCK_LEAN = 12
SSORT_PARAM_MATCH_VOTE = 13
SSORT_PARAM_WARP_MERGE = 14
SSORT_PARAM_SCAN = 15


class SsortError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__(f"ssort status {status}: {msg}")
        self.status = status


class Stats(ctypes.Structure):
    _fields_ = [
        ("n", ctypes.c_uint64),
        ("rounds", ctypes.c_uint32),
        ("partition_levels", ctypes.c_uint32),
        ("live", ctypes.c_uint64 * SSORT_MAX_ROUNDS),
        ("partitioned", ctypes.c_uint64),
        ("small_segments", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
        ("device_ms", ctypes.c_double),
        ("gather_elems", ctypes.c_uint64),
        ("warp1_fresh", ctypes.c_uint64),
        ("warp1_keyed", ctypes.c_uint64),
        ("warp8_fresh", ctypes.c_uint64),
        ("warp8_keyed", ctypes.c_uint64),
        ("block_fresh", ctypes.c_uint64),
        ("block_keyed", ctypes.c_uint64),
        ("equal_moved", ctypes.c_uint64),
        ("equal_final", ctypes.c_uint64),
        ("boundaries", ctypes.c_uint64),
        ("gather_fused", ctypes.c_uint64),
        ("warp1_deep", ctypes.c_uint64),
        ("full_sorted", ctypes.c_uint64),
        ("window_saved", ctypes.c_uint64),
        ("window_used", ctypes.c_uint64),
        ("graph_launches", ctypes.c_uint64),
    ]

    def as_dict(self):
        d = {f: getattr(self, f) for f, _ in self._fields_ if f != "live"}
        d["live"] = [int(self.live[i]) for i in range(min(self.rounds, SSORT_MAX_ROUNDS))]
        return d


class ServerInfo(ctypes.Structure):
    _fields_ = [
        ("queued", ctypes.c_uint32),
        ("loading", ctypes.c_uint32),
        ("active", ctypes.c_uint32),
        ("draining", ctypes.c_uint32),
        ("max_active", ctypes.c_uint32),
        ("rounds", ctypes.c_uint64),
        ("requests_done", ctypes.c_uint64),
        ("strings_done", ctypes.c_uint64),
        ("arena_in_use", ctypes.c_uint64),
        ("strings_in_use", ctypes.c_uint64),
        ("arena_budget", ctypes.c_uint64),
        ("max_strings", ctypes.c_uint64),
        ("device_bytes", ctypes.c_uint64),
    ]

    def as_dict(self):
        return {f: int(getattr(self, f)) for f, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [
        ("size_class", ctypes.c_uint32),
        ("entropy_class", ctypes.c_uint32),
        ("entropy_bits", ctypes.c_double),
        ("target_bucket", ctypes.c_int64),
        ("warp8_cap", ctypes.c_int64),
        ("overlap", ctypes.c_int64),
        ("fused_gather", ctypes.c_int64),
        ("default_ms", ctypes.c_double),
        ("tuned_ms", ctypes.c_double),
        ("trials", ctypes.c_uint32),
        ("digit_bits", ctypes.c_int64),
        ("block_prefetch", ctypes.c_int64),
        ("l2_prefetch", ctypes.c_int64),
        ("graph", ctypes.c_int64),
    ]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None
_wlib = None


def lib():
    """Load libssort_b200.so (raises if it was not built)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with string-sorting_b200/build.py")
        L = ctypes.CDLL(LIB_PATH)
        vp, u64, i32 = ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int
        L.ssort_strerror.restype = ctypes.c_char_p
        L.ssort_strerror.argtypes = [i32]
        L.ssort_last_error.restype = ctypes.c_char_p
        L.ssort_last_error.argtypes = []
        L.ssort_ctx_create.argtypes = [i32, ctypes.POINTER(vp)]
        L.ssort_ctx_destroy.argtypes = [vp]
        L.ssort_ctx_destroy.restype = None
        L.ssort_sort_device.argtypes = [vp, vp, u64, vp, i32, u64, vp, vp, vp]
        L.ssort_sort_device_noalloc.argtypes = [vp, u64, vp, i32, u64, vp, vp, vp]
        L.ssort_sort_host.argtypes = [vp, vp, u64, vp, i32, u64, vp, vp]
        L.ssort_sort_strings.argtypes = [vp, vp, ctypes.c_size_t, vp]
        L.ssort_get_stats.argtypes = [vp, ctypes.POINTER(Stats)]
        L.ssort_set_profiling.argtypes = [vp, i32]
        L.ssort_set_param.argtypes = [vp, i32, ctypes.c_int64]
        L.ssort_sort_batch_device.argtypes = [vp, vp, u64, vp, i32, u64, vp, ctypes.c_uint32,
                                              vp, vp, vp]
        L.ssort_sort_batch_host.argtypes = [vp, vp, u64, vp, i32, u64, vp, ctypes.c_uint32,
                                            vp, vp]
        L.ssort_get_kernel_times.argtypes = [vp, ctypes.POINTER(ctypes.c_char_p),
                                             ctypes.POINTER(ctypes.c_double),
                                             ctypes.POINTER(ctypes.c_uint64), i32]
        L.ssort_server_create.argtypes = [i32, u64, u64, ctypes.POINTER(vp)]
        L.ssort_server_destroy.argtypes = [vp]
        L.ssort_server_destroy.restype = None
        L.ssort_server_submit.argtypes = [vp, vp, u64, vp, i32, u64, vp, vp,
                                          ctypes.POINTER(u64)]
        L.ssort_server_step.argtypes = [vp, ctypes.POINTER(u64), ctypes.c_uint32,
                                        ctypes.POINTER(ctypes.c_uint32)]
        L.ssort_server_poll.argtypes = [vp, u64, ctypes.POINTER(i32)]
        L.ssort_server_drain.argtypes = [vp]
        L.ssort_server_get_info.argtypes = [vp, ctypes.POINTER(ServerInfo)]
        L.ssort_text_offsets_device.argtypes = [vp, vp, u64, i32, vp, i32, u64,
                                                ctypes.POINTER(u64), vp]
        L.ssort_sort_text_host.argtypes = [vp, vp, u64, i32, vp, vp, u64, ctypes.POINTER(u64)]
        L.ssort_merge_runs.argtypes = [vp, u64, vp, i32, u64, vp, ctypes.c_uint32, vp, vp, vp,
                                       vp]
        L.ssort_sort_host_chunked.argtypes = [vp, vp, u64, vp, i32, u64, u64, vp, vp]
        L.ssort_autotune.argtypes = [vp, vp, u64, vp, i32, u64, ctypes.POINTER(Tuning)]
        L.ssort_pinned_alloc.argtypes = [ctypes.c_size_t, ctypes.POINTER(vp)]
        L.ssort_pinned_free.argtypes = [vp]
        L.ssort_pinned_free.restype = None
        L.msd_gpu.argtypes = [vp, ctypes.c_size_t]
        L.msd_gpu.restype = None
        _lib = L
    return _lib


def _check(status):
    if status != SSORT_OK:
        L = lib()
        raise SsortError(status, f"{L.ssort_strerror(status).decode()}: "
                                 f"{L.ssort_last_error().decode()}")


def _ptr(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data
    return a.data_ptr()  # torch tensor


class Sorter:
    """One sort context (a CUDA stream plus a reusable device workspace)."""

    def __init__(self, device=0):
        self._ctx = ctypes.c_void_p()
        _check(lib().ssort_ctx_create(int(device), ctypes.byref(self._ctx)))

    def close(self):
        if self._ctx:
            lib().ssort_ctx_destroy(self._ctx)
            self._ctx = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- entry points ---------------------------------------------------------
    def sort_host(self, arena, offs, with_lcp=True, perm=None, lcp=None):
        """Sort from host buffers (numpy): arena uint8, offs uint32/uint64."""
        arena = np.ascontiguousarray(arena, dtype=np.uint8)
        offs = np.ascontiguousarray(offs)
        if offs.dtype not in (np.uint32, np.uint64):
            raise TypeError("offsets must be uint32 or uint64")
        n = offs.shape[0]
        if perm is None:
            perm = np.empty(n, dtype=np.uint32)
        if with_lcp and lcp is None:
            lcp = np.empty(n, dtype=np.uint32)
        _check(lib().ssort_sort_host(self._ctx, _ptr(arena), arena.nbytes, _ptr(offs),
                                     offs.dtype.itemsize, n, _ptr(perm),
                                     _ptr(lcp) if with_lcp else None))
        return perm, (lcp if with_lcp else None)

    def sort_device(self, d_arena, arena_bytes, d_offs, off_width, n, d_perm, d_lcp=None,
                    stream=None):
        """Sort device-resident buffers (torch CUDA tensors or raw pointers)."""
        def p(x):
            return x if isinstance(x, int) or x is None else x.data_ptr()
        _check(lib().ssort_sort_device(self._ctx, p(d_arena), int(arena_bytes), p(d_offs),
                                       int(off_width), int(n), p(d_perm), p(d_lcp),
                                       stream))

    def sort_batch_host(self, arena, offs, inst_start, with_lcp=True, perm=None, lcp=None):
        """Batched sort from host buffers: inst_start (uint32, ninst + 1 entries)
        splits the offsets into independent instances; perm is instance-local."""
        arena = np.ascontiguousarray(arena, dtype=np.uint8)
        offs = np.ascontiguousarray(offs)
        inst = np.ascontiguousarray(inst_start, dtype=np.uint32)
        n = offs.shape[0]
        if perm is None:
            perm = np.empty(n, dtype=np.uint32)
        if with_lcp and lcp is None:
            lcp = np.empty(n, dtype=np.uint32)
        _check(lib().ssort_sort_batch_host(self._ctx, _ptr(arena), arena.nbytes, _ptr(offs),
                                           offs.dtype.itemsize, n, _ptr(inst), inst.shape[0] - 1,
                                           _ptr(perm), _ptr(lcp) if with_lcp else None))
        return perm, (lcp if with_lcp else None)

    def sort_batch_device(self, d_arena, arena_bytes, d_offs, off_width, n, d_inst, ninst,
                          d_perm, d_lcp=None, stream=None):
        """Batched sort of device-resident buffers (torch tensors or pointers)."""
        def p(x):
            return x if isinstance(x, int) or x is None else x.data_ptr()
        _check(lib().ssort_sort_batch_device(self._ctx, p(d_arena), int(arena_bytes), p(d_offs),
                                             int(off_width), int(n), p(d_inst), int(ninst),
                                             p(d_perm), p(d_lcp), stream))

    def sort_strings(self, strings, with_lcp=False):
        """Pointer-array form: strings is a list of bytes objects (no NULs).
        Returns the sorted list (and the LCP array)."""
        n = len(strings)
        bufs = [ctypes.create_string_buffer(s) for s in strings]
        arr = (ctypes.c_void_p * max(n, 1))(*[ctypes.addressof(b) for b in bufs])
        lcp = np.empty(n, dtype=np.uint32) if with_lcp else None
        _check(lib().ssort_sort_strings(self._ctx, arr, n, _ptr(lcp)))
        addr = {ctypes.addressof(b): i for i, b in enumerate(bufs)}
        order = [addr[arr[i]] for i in range(n)]
        out = [strings[i] for i in order]
        return (out, lcp) if with_lcp else out

    def sort_host_chunked(self, arena, offs, chunk, with_lcp=True):
        """Sort with a workspace for `chunk` strings: GPU-sorted chunks merged
        on the host by their LCPs."""
        arena = np.ascontiguousarray(arena, dtype=np.uint8)
        offs = np.ascontiguousarray(offs)
        n = offs.shape[0]
        perm = np.empty(n, dtype=np.uint32)
        lcp = np.empty(n, dtype=np.uint32) if with_lcp else None
        _check(lib().ssort_sort_host_chunked(self._ctx, _ptr(arena), arena.nbytes, _ptr(offs),
                                             offs.dtype.itemsize, n, int(chunk), _ptr(perm),
                                             _ptr(lcp)))
        return perm, lcp

    def sort_text(self, text, mode=TEXT_LINES, with_lcp=True, out=None, lcp=None):
        """Sort the strings of a whole text (bytes or uint8 array) as sortstring
        makes them; returns (sorted string starts as uint64 offsets, lcp).
        With `out` given (uint64, one entry per string, and `lcp` likewise when
        with_lcp) the call writes there and skips the sizing call."""
        buf = np.frombuffer(text, dtype=np.uint8) if isinstance(text, (bytes, bytearray)) \
            else np.ascontiguousarray(text, dtype=np.uint8)
        L = lib()
        n = ctypes.c_uint64()
        if out is None:
            rc = L.ssort_sort_text_host(self._ctx, _ptr(buf), buf.nbytes, int(mode), None, None,
                                        0, ctypes.byref(n))
            if rc != SSORT_OK and n.value == 0:
                _check(rc)
            out = np.empty(n.value, dtype=np.uint64)
        if with_lcp and lcp is None:
            lcp = np.empty(len(out), dtype=np.uint32)
        if not with_lcp:
            lcp = None
        _check(L.ssort_sort_text_host(self._ctx, _ptr(buf), buf.nbytes, int(mode), _ptr(out),
                                      _ptr(lcp), len(out), ctypes.byref(n)))
        return out[:n.value], lcp[:n.value] if lcp is not None else None

    def text_offsets_device(self, d_text, text_len, mode, d_offs, off_width, cap, stream=None):
        """String starts of a device-resident text (torch tensors or
        addresses); returns the number of strings."""
        def p(x):
            return x if isinstance(x, int) or x is None else x.data_ptr()
        n = ctypes.c_uint64()
        _check(lib().ssort_text_offsets_device(self._ctx, p(d_text), int(text_len), int(mode),
                                               p(d_offs), int(off_width), int(cap),
                                               ctypes.byref(n), stream))
        return n.value

    def stats(self):
        s = Stats()
        _check(lib().ssort_get_stats(self._ctx, ctypes.byref(s)))
        return s

    def set_param(self, param, value):
        _check(lib().ssort_set_param(self._ctx, int(param), int(value)))

    def autotune(self, d_arena, arena_bytes, d_offs, off_width, n):
        """Tune the context's parameters on a device-resident input
        (ssort_autotune); returns the chosen values and timings."""
        def p(x):
            return x if isinstance(x, int) or x is None else x.data_ptr()
        t = Tuning()
        _check(lib().ssort_autotune(self._ctx, p(d_arena), int(arena_bytes), p(d_offs),
                                    int(off_width), int(n), ctypes.byref(t)))
        return t.as_dict()

    def set_profiling(self, on):
        _check(lib().ssort_set_profiling(self._ctx, 1 if on else 0))

    def kernel_times(self):
        L = lib()
        k = L.ssort_get_kernel_times(self._ctx, None, None, None, 0)
        names = (ctypes.c_char_p * max(k, 1))()
        ms = (ctypes.c_double * max(k, 1))()
        cnt = (ctypes.c_uint64 * max(k, 1))()
        L.ssort_get_kernel_times(self._ctx, names, ms, cnt, k)
        return {names[i].decode(): (ms[i], cnt[i]) for i in range(k)}


def merge_runs(arena, offs, run_start, perm, lcp):
    """Host LCP merge of sorted runs (ssort_merge_runs): perm/lcp hold each
    run's run-local result; returns the global (perm, lcp)."""
    arena = np.ascontiguousarray(arena, dtype=np.uint8)
    offs = np.ascontiguousarray(offs)
    rs = np.ascontiguousarray(run_start, dtype=np.uint32)
    perm = np.ascontiguousarray(perm, dtype=np.uint32)
    lcp = np.ascontiguousarray(lcp, dtype=np.uint32)
    n = offs.shape[0]
    out_p = np.empty(n, dtype=np.uint32)
    out_l = np.empty(n, dtype=np.uint32)
    _check(lib().ssort_merge_runs(_ptr(arena), arena.nbytes, _ptr(offs), offs.dtype.itemsize, n,
                                  _ptr(rs), rs.shape[0] - 1, _ptr(perm), _ptr(lcp),
                                  _ptr(out_p), _ptr(out_l)))
    return out_p, out_l


class Server:
    """Request server: sort requests from host buffers, batched between rounds
    (ssort_server_* in include/ssort_b200.h).  The buffers of each request are
    kept referenced here until the request is reported done."""

    def __init__(self, arena_budget, max_strings, device=0):
        self._srv = ctypes.c_void_p()
        _check(lib().ssort_server_create(int(device), int(arena_budget), int(max_strings),
                                         ctypes.byref(self._srv)))
        self._held = {}
        self._ids = (ctypes.c_uint64 * 4096)()

    def close(self):
        if self._srv:
            lib().ssort_server_destroy(self._srv)
            self._srv = ctypes.c_void_p()
            self._held.clear()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def submit(self, arena, offs, perm=None, lcp=None, with_lcp=True):
        """Queue one request; returns (id, perm, lcp) with perm/lcp filled once
        the request is done.  arena (uint8) and offs (uint32/uint64) are numpy
        arrays, ideally in pinned memory."""
        arena = np.ascontiguousarray(arena, dtype=np.uint8)
        offs = np.ascontiguousarray(offs)
        if offs.dtype not in (np.uint32, np.uint64):
            raise TypeError("offsets must be uint32 or uint64")
        n = offs.shape[0]
        if perm is None:
            perm = np.empty(n, dtype=np.uint32)
        if with_lcp and lcp is None:
            lcp = np.empty(n, dtype=np.uint32)
        rid = ctypes.c_uint64()
        _check(lib().ssort_server_submit(self._srv, _ptr(arena), arena.nbytes, _ptr(offs),
                                         offs.dtype.itemsize, n, _ptr(perm),
                                         _ptr(lcp) if with_lcp else None, ctypes.byref(rid)))
        self._held[rid.value] = (arena, offs, perm, lcp)
        return rid.value, perm, (lcp if with_lcp else None)

    def submit_ptr(self, arena, arena_bytes, offs, off_width, n, perm, lcp=None):
        """Queue one request given raw addresses or torch tensors, in host
        memory or in device memory of the server's device; returns its id."""
        def p(x):
            return x if isinstance(x, int) or x is None else x.data_ptr()
        rid = ctypes.c_uint64()
        _check(lib().ssort_server_submit(self._srv, p(arena), int(arena_bytes), p(offs),
                                         int(off_width), int(n), p(perm), p(lcp),
                                         ctypes.byref(rid)))
        self._held[rid.value] = (arena, offs, perm, lcp)
        return rid.value

    def step(self):
        """One scheduling step; returns the ids completed since the last step."""
        k = ctypes.c_uint32()
        _check(lib().ssort_server_step(self._srv, self._ids, len(self._ids), ctypes.byref(k)))
        done = [int(self._ids[i]) for i in range(k.value)]
        for rid in done:
            self._held.pop(rid, None)
        return done

    def poll(self, rid):
        st = ctypes.c_int()
        _check(lib().ssort_server_poll(self._srv, int(rid), ctypes.byref(st)))
        return st.value

    def drain(self):
        """Run until every submitted request is done; returns their ids."""
        _check(lib().ssort_server_drain(self._srv))
        done = []
        while True:
            got = self.step()
            if not got:
                break
            done += got
        return done

    def info(self):
        i = ServerInfo()
        _check(lib().ssort_server_get_info(self._srv, ctypes.byref(i)))
        return i.as_dict()


# ---- synthetic workloads ------------------------------------------------------
class StringSet:
    """An arena of NUL-terminated strings plus uint64 offsets, owned by the
    workload library (freed on garbage collection)."""

    def __init__(self, arena_ptr, arena_bytes, offs_ptr, n):
        self._arena_ptr = arena_ptr
        self._offs_ptr = offs_ptr
        self.n = int(n)
        self.text_bytes = int(arena_bytes)  # without the 16 padding bytes
        ab = arena_bytes + 16
        self.arena = np.ctypeslib.as_array(
            ctypes.cast(arena_ptr, ctypes.POINTER(ctypes.c_uint8)), shape=(ab,))
        self.offs = np.ctypeslib.as_array(
            ctypes.cast(offs_ptr, ctypes.POINTER(ctypes.c_uint64)), shape=(max(self.n, 1),))[:self.n]

    def __del__(self):
        try:
            if self._arena_ptr:
                wlib().ssw_free(self._arena_ptr)
                wlib().ssw_free(self._offs_ptr)
                self._arena_ptr = None
        except Exception:
            pass

    def string(self, i):
        o = int(self.offs[i])
        e = o
        while self.arena[e] != 0:
            e += 1
        return bytes(self.arena[o:e])

    def key_bytes(self):
        """Sum of (length + 1) over all strings: the bytes the sort keys on."""
        return self.text_bytes


def wlib():
    global _wlib
    if _wlib is None:
        if not os.path.exists(WLIB_PATH):
            raise FileNotFoundError(f"{WLIB_PATH} is missing: build string-sorting_b200/build.py")
        W = ctypes.CDLL(WLIB_PATH)
        pp8 = ctypes.POINTER(ctypes.c_void_p)
        u64p = ctypes.POINTER(ctypes.c_uint64)
        W.ssw_gen_uniform.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32,
                                      ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64,
                                      pp8, u64p, pp8]
        W.ssw_gen_urls.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                                   ctypes.c_uint64, pp8, u64p, pp8]
        W.ssw_gen_zipf_words.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_double,
                                         ctypes.c_uint32, ctypes.c_double, ctypes.c_uint64,
                                         pp8, u64p, pp8]
        W.ssw_gen_instances.argtypes = [ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64,
                                        ctypes.c_void_p, pp8, u64p, pp8]
        W.ssw_free.argtypes = [ctypes.c_void_p]
        W.ssw_free.restype = None
        W.ssw_uniform_doubles.argtypes = [ctypes.c_uint64, ctypes.c_uint64,
                                          ctypes.POINTER(ctypes.c_double)]
        W.ssw_uniform_doubles.restype = None
        _wlib = W
    return _wlib


def _gen(fn, *args):
    a = ctypes.c_void_p()
    o = ctypes.c_void_p()
    nb = ctypes.c_uint64()
    rc = fn(*args, ctypes.byref(a), ctypes.byref(nb), ctypes.byref(o))
    if rc != 0:
        raise RuntimeError(f"workload generator failed ({rc})")
    return a.value, nb.value, o.value


def gen_uniform(n, min_len=1, max_len=20, alpha_lo=ord("a"), alpha_size=26, seed=1):
    a, nb, o = _gen(wlib().ssw_gen_uniform, n, min_len, max_len, alpha_lo, alpha_size, seed)
    return StringSet(a, nb, o, n)


def gen_urls(n, n_hosts=4096, zipf_s=1.1, seed=2):
    a, nb, o = _gen(wlib().ssw_gen_urls, n, n_hosts, zipf_s, seed)
    return StringSet(a, nb, o, n)


def gen_zipf_words(n, vocab=1_000_000, p_geom=0.15, max_len=24, zipf_s=1.0, seed=3):
    a, nb, o = _gen(wlib().ssw_gen_zipf_words, n, vocab, p_geom, max_len, zipf_s, seed)
    return StringSet(a, nb, o, n)


def gen_repeat_text(nbytes, n_repeats=2000, min_rep=32, max_rep=4096, seed=8):
    """A text of nbytes bytes for suffix sorting: Zipf(1.0) words (as
    gen_zipf_words, seed `seed`) separated by single spaces, then n_repeats
    passages of log-uniform length in [min_rep, max_rep] copied from a uniform
    position to another (the long repeats of real corpora, which make suffix
    LCPs deep).  Returns a uint8 array: the text followed by 16 zero bytes."""
    words = gen_zipf_words(nbytes // 7 + 64, seed=seed)  # >= 8 bytes per word on average
    if words.text_bytes < nbytes:
        raise ValueError("word text shorter than requested")
    text = np.zeros(nbytes + 16, dtype=np.uint8)
    text[:nbytes] = words.arena[:nbytes]
    body = text[:nbytes]
    body[body == 0] = ord(" ")
    rng = np.random.default_rng(seed)
    lens = np.exp(rng.uniform(np.log(min_rep), np.log(max_rep), size=n_repeats)).astype(np.int64)
    lens = np.minimum(lens, nbytes // 2)
    for L in lens:
        a, b = rng.integers(0, nbytes - L, size=2)
        body[b:b + L] = body[a:a + L].copy()
    return text


class InstanceSet(StringSet):
    """Several independent sort instances in one arena; inst_start has
    ninst + 1 entries (position ranges of the instances)."""

    def __init__(self, arena_ptr, arena_bytes, offs_ptr, n, inst_start, params):
        super().__init__(arena_ptr, arena_bytes, offs_ptr, n)
        self.inst_start = inst_start
        self.params = params  # per instance: (count, max_len, alpha_lo, alpha_size)

    def request(self, i, off_dtype=np.uint32):
        """Instance i as a stand-alone request: (arena view, offsets relative
        to it).  The instance's strings are contiguous in the shared arena."""
        lo, hi = int(self.inst_start[i]), int(self.inst_start[i + 1])
        if hi == lo:
            return self.arena[:0], np.zeros(0, dtype=off_dtype)
        a0 = int(self.offs[lo])
        a1 = int(self.offs[hi]) if hi < self.n else self.text_bytes
        return self.arena[a0:a1], (self.offs[lo:hi] - np.uint64(a0)).astype(off_dtype)


# Per-instance shapes of the batched workload: alphabets of 4 from 'A', 26
# from 'a', 95 from ' '; length bounds 8, 32, 128.
BATCH_ALPHABETS = ((ord("A"), 4), (ord("a"), 26), (ord(" "), 95))
BATCH_MAX_LENS = (8, 32, 128)


def batch_instance_params(ninst, seed, lo=100, hi=2_000_000, key_byte_limit=None):
    """Instance parameters of the batched workload: string counts log-uniform
    in [lo, hi], alphabet and length bound drawn uniformly from the sets
    above.  With key_byte_limit, the list stops once the expected key bytes
    (count * (mean length + 1)) reach the limit."""
    import math
    u = uniform_doubles(3 * ninst, seed)
    out, total = [], 0.0
    for k in range(ninst):
        count = int(round(math.exp(math.log(lo) + u[3 * k] * (math.log(hi) - math.log(lo)))))
        a_lo, a_sz = BATCH_ALPHABETS[min(2, int(u[3 * k + 1] * 3))]
        L = BATCH_MAX_LENS[min(2, int(u[3 * k + 2] * 3))]
        out.append((count, L, a_lo, a_sz))
        total += count * ((1 + L) / 2 + 1)
        if key_byte_limit is not None and total >= key_byte_limit:
            break
    return out


def gen_instances(params, seed=4):
    """Generate the instances described by batch_instance_params."""
    k = len(params)
    counts = np.array([p[0] for p in params], dtype=np.uint64)
    lens = np.array([p[1] for p in params], dtype=np.uint32)
    alo = np.array([p[2] for p in params], dtype=np.uint32)
    asz = np.array([p[3] for p in params], dtype=np.uint32)
    inst = np.zeros(k + 1, dtype=np.uint32)
    a = ctypes.c_void_p()
    o = ctypes.c_void_p()
    nb = ctypes.c_uint64()
    rc = wlib().ssw_gen_instances(k, counts.ctypes.data, lens.ctypes.data, alo.ctypes.data,
                                  asz.ctypes.data, seed, inst.ctypes.data, ctypes.byref(a),
                                  ctypes.byref(nb), ctypes.byref(o))
    if rc != 0:
        raise RuntimeError(f"instance generator failed ({rc})")
    return InstanceSet(a.value, nb.value, o.value, int(counts.sum()), inst, params)


def uniform_doubles(n, seed):
    out = np.empty(n, dtype=np.float64)
    wlib().ssw_uniform_doubles(n, seed, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)))
    return out


# The workloads the benchmark and the parity tests use, by name.
WORKLOADS = {
    # 1,000,000 strings, length U[1,20], bytes U{'a'..'z'}, seed 1
    "uniform_1m": lambda scale=1.0: gen_uniform(int(1_000_000 * scale), 1, 20, ord("a"), 26, 1),
    # 50,000,000 URLs: "http://" + Zipf(1.1) host of 4096 + 1..6 path segments
    "urls_50m": lambda scale=1.0: gen_urls(int(50_000_000 * scale), 4096, 1.1, 2),
    # 100,000,000 copies of Zipf(1.0) words from a 1,000,000-word vocabulary
    "zipf_words_100m": lambda scale=1.0: gen_zipf_words(int(100_000_000 * scale), 1_000_000,
                                                        0.15, 24, 1.0, 3),
}
