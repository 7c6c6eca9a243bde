"""ctypes binding of the b200sort C ABI (include/b200sort.h).

The library is the product; this module only loads it and forwards calls.
There is no fallback: if libb200sort.so is missing the import of `lib()`
raises, and every sort runs the CUDA kernels of that library.

Device buffers are passed as integer device pointers (for example
`tensor.data_ptr()` of a CUDA tensor) and streams as integer cudaStream_t
handles (for example `torch.cuda.current_stream().cuda_stream`).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# B200SORT_LIB names another build of the library (for example an experimental
# one); its tile table is read from tune/b200_table.csv beside it.
LIB_PATH = os.environ.get("B200SORT_LIB", os.path.join(HERE, "libb200sort.so"))

I32, I32_I32, U64, U64_I32 = 0, 1, 2, 3
DTYPES = {"i32": I32, "i32_i32": I32_I32, "u64": U64, "u64_i32": U64_I32}
STABLE = 1
SORTED_CHECK = 2
PLAN_NO_GRAPH = 0x100
ELEM_BYTES = {I32: 4, I32_I32: 8, U64: 8, U64_I32: 16}

# numpy views of the memory layouts
NP_DTYPES = {
    I32: np.dtype("<i4"),
    I32_I32: np.dtype([("key", "<i4"), ("data", "<i4")]),
    U64: np.dtype("<u8"),
    U64_I32: np.dtype([("key", "<u8"), ("data", "<i4"), ("reserved", "<i4")]),
}

OK = 0
STATUS_NAMES = {0: "OK", 1: "INVALID_ARGUMENT", 2: "UNSUPPORTED", 3: "CUDA", 4: "OUT_OF_MEMORY",
                5: "TIMEOUT", 6: "BUDGET", 7: "BUSY", 8: "CANCELLED"}
ERR_TIMEOUT, ERR_BUDGET, ERR_BUSY, ERR_CANCELLED = 5, 6, 7, 8
MEM_DEVICE, MEM_HOST = 0, 1
REQ_FREE, REQ_QUEUED, REQ_RUNNING, REQ_DONE, REQ_FAILED, REQ_CANCELLED = range(6)


class Tile(ctypes.Structure):
    _fields_ = [("log2_items", ctypes.c_int32), ("log2_lanes", ctypes.c_int32),
                ("log2_warps", ctypes.c_int32), ("cta_threads", ctypes.c_int32),
                ("persistent", ctypes.c_int32), ("log2_ctas", ctypes.c_int32)]

    def as_tuple(self):
        return (self.log2_items, self.log2_lanes, self.log2_warps, self.log2_ctas)

    def __repr__(self):
        return "Tile(K=%d, lanes=%d, warps=%d, ctas=%d, cta=%d, form=%d)" % (
            1 << self.log2_items, 1 << self.log2_lanes, 1 << self.log2_warps, 1 << self.log2_ctas,
            self.cta_threads, self.persistent)

    def with_persistent(self, on=True):
        return Tile(self.log2_items, self.log2_lanes, self.log2_warps, self.cta_threads, 1 if on else 0,
                    self.log2_ctas)

    def with_form(self, form):
        """The same shape with launch form 0 (one-shot), 1 (register prefetch), 2 (TMA pipeline) or 3
        (transposed network)."""
        return Tile(self.log2_items, self.log2_lanes, self.log2_warps, self.cta_threads, form, self.log2_ctas)


class TileInfo(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int32) for n in ("registers_per_thread", "local_bytes_per_thread", "shared_bytes",
                                              "cta_threads", "active_ctas_per_sm", "working", "arrays_per_cta",
                                              "tma_form", "xpose_form")]


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int32), ("dtype", ctypes.c_int), ("flags", ctypes.c_uint32),
                ("budget_bytes", ctypes.c_int64), ("max_inflight", ctypes.c_int32), ("max_batch", ctypes.c_int32),
                ("max_queue", ctypes.c_int64)]


class ServerStats(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int64) for n in (
        "submitted", "completed", "failed", "cancelled", "rejected", "batches", "keys_completed", "queued",
        "inflight_batches", "peak_arena_bytes", "arena_bytes", "max_batch_requests")] + \
        [(n, ctypes.c_double) for n in ("mean_batch_requests", "p50_us", "p99_us", "p999_us", "max_us", "mean_us",
                                        "span_s")]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_}


class B200SortError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("b200sort %s: %s" % (STATUS_NAMES.get(status, status), message))
        self.status = status


_lib = None

_SIGNATURES = {
    "b200s_version": (ctypes.c_char_p, []),
    "b200s_status_string": (ctypes.c_char_p, [ctypes.c_int]),
    "b200s_last_error": (ctypes.c_char_p, []),
    "b200s_max_length": (ctypes.c_int32, [ctypes.c_int, ctypes.c_uint32]),
    "b200s_tile_count": (ctypes.c_int32, [ctypes.c_int, ctypes.c_uint32]),
    "b200s_tile_get": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint32, ctypes.c_int32, ctypes.POINTER(Tile)]),
    "b200s_default_tile": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint32, ctypes.c_int32, ctypes.POINTER(Tile)]),
    "b200s_tile_info_get": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint32, ctypes.POINTER(Tile), ctypes.c_int32,
                                           ctypes.POINTER(TileInfo)]),
    "b200s_load_tile_table": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32)]),
    "b200s_sort_packed": (ctypes.c_int, [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                         ctypes.c_int64, ctypes.c_uint32, ctypes.POINTER(Tile),
                                         ctypes.c_void_p]),
    "b200s_plan_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_uint32,
                                         ctypes.c_int64, ctypes.c_int32]),
    "b200s_plan_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "b200s_ragged_max_length": (ctypes.c_int32, [ctypes.c_int, ctypes.c_uint32]),
    "b200s_sort_ragged": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                         ctypes.c_int64, ctypes.c_void_p]),
    "b200s_sort_ragged_hinted": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                                ctypes.c_void_p, ctypes.c_int64, ctypes.c_void_p]),
    "b200s_plan_too_long": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.POINTER(ctypes.c_int64)]),
    "b200s_plan_prepare_plain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]),
    "b200s_sort_ragged_plain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                               ctypes.c_void_p, ctypes.c_void_p]),
    "b200s_plan_plain_launches": (ctypes.c_int32, [ctypes.c_void_p]),
    "b200s_plan_prepare_plain_buckets": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64]),
    "b200s_sort_partitions": (ctypes.c_int, [ctypes.c_int, ctypes.c_uint32, ctypes.c_void_p, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p]),
    "b200s_release_partition_plans": (ctypes.c_int, []),
    "b200s_session_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int32]),
    "b200s_session_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "b200s_sort_packed_host": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                              ctypes.c_int32, ctypes.c_int64, ctypes.c_uint32]),
    "b200s_server_create": (ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.POINTER(ServerConfig)]),
    "b200s_server_destroy": (ctypes.c_int, [ctypes.c_void_p]),
    "b200s_server_submit": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                           ctypes.c_uint32, ctypes.POINTER(ctypes.c_uint64)]),
    "b200s_server_submit_arrived": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32,
                                                   ctypes.c_uint32, ctypes.c_int64, ctypes.POINTER(ctypes.c_uint64)]),
    "b200s_server_clock_ns": (ctypes.c_int64, []),
    "b200s_server_wait": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.c_int64,
                                         ctypes.POINTER(ctypes.c_int)]),
    "b200s_server_poll": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_int32),
                                         ctypes.POINTER(ctypes.c_int)]),
    "b200s_server_cancel": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_uint64]),
    "b200s_server_drain": (ctypes.c_int, [ctypes.c_void_p, ctypes.c_int64]),
    "b200s_server_stats_get": (ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ServerStats), ctypes.c_int32]),
}


def lib():
    """Load libb200sort.so once and declare the C signatures."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError("libb200sort.so not built at %s (run __graft_entry__.build())" % LIB_PATH)
        handle = ctypes.CDLL(LIB_PATH)
        for name, (res, args) in _SIGNATURES.items():
            fn = getattr(handle, name)
            fn.restype = res
            fn.argtypes = args
        _lib = handle
    return _lib


def declare(name, restype, argtypes):
    """Declare an additional entry point of the library (used by sibling modules)."""
    fn = getattr(lib(), name)
    fn.restype = restype
    fn.argtypes = argtypes
    return fn


def check(status):
    if status != OK:
        raise B200SortError(status, lib().b200s_last_error().decode())
    return status


def version():
    return lib().b200s_version().decode()


def max_length(dtype, flags=0):
    return lib().b200s_max_length(dtype, flags)


def tiles(dtype, flags=0):
    out = []
    for i in range(lib().b200s_tile_count(dtype, flags)):
        t = Tile()
        check(lib().b200s_tile_get(dtype, flags, i, ctypes.byref(t)))
        out.append(t)
    return out


def default_tile(dtype, n, flags=0):
    t = Tile()
    check(lib().b200s_default_tile(dtype, flags, n, ctypes.byref(t)))
    return t


def tile_info(dtype, n, flags=0, tile=None):
    """Registers, local memory, shared memory and residency of the kernel for length n."""
    out = TileInfo()
    check(lib().b200s_tile_info_get(dtype, flags, ctypes.byref(tile) if tile is not None else None, n,
                                    ctypes.byref(out)))
    return out


def load_tile_table(path):
    applied = ctypes.c_int32(0)
    check(lib().b200s_load_tile_table(path.encode(), ctypes.byref(applied)))
    return applied.value


def sort_packed(dtype, d_in, d_out, n, arrays, flags=0, tile=None, stream=0):
    """Sort `arrays` packed arrays of n elements from device pointer d_in to d_out."""
    tp = ctypes.byref(tile) if tile is not None else None
    return check(lib().b200s_sort_packed(dtype, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), n, arrays,
                                         flags, tp, ctypes.c_void_p(stream)))


def sort_partitions(dtype, d_in, d_out, d_counters, nb_parts, d_uniform=0, flags=0, stream=0):
    """Sort every partition [counters[p], counters[p+1]) of a partitioned array
    (the leaf of the reference's large-array sort), device pointers."""
    return check(lib().b200s_sort_partitions(dtype, flags, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                                             ctypes.c_void_p(d_counters), ctypes.c_void_p(d_uniform or None),
                                             nb_parts, ctypes.c_void_p(stream)))


def sort_packed_status(dtype, d_in, d_out, n, arrays, flags=0, tile=None, stream=0):
    """Like sort_packed but returns the raw status code instead of raising."""
    tp = ctypes.byref(tile) if tile is not None else None
    return lib().b200s_sort_packed(dtype, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out), n, arrays, flags,
                                   tp, ctypes.c_void_p(stream))


class Session:
    """Host-buffer sorting: copies in, sorts on the device, copies out."""

    def __init__(self, device=0):
        self._h = ctypes.c_void_p()
        check(lib().b200s_session_create(ctypes.byref(self._h), device))

    def sort_host(self, dtype, h_in, h_out, n, arrays, flags=0):
        return check(lib().b200s_sort_packed_host(self._h, dtype, ctypes.c_void_p(h_in), ctypes.c_void_p(h_out),
                                                  n, arrays, flags))

    def close(self):
        if self._h:
            lib().b200s_session_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ragged_max_length(dtype, flags=0):
    return lib().b200s_ragged_max_length(dtype, flags)


class Plan:
    """A ragged-batch plan: scratch for max_arrays arrays and a captured CUDA graph."""

    def __init__(self, dtype, max_arrays, flags=0, device=0):
        self.dtype = dtype
        self._h = ctypes.c_void_p()
        check(lib().b200s_plan_create(ctypes.byref(self._h), dtype, flags, max_arrays, device))

    def sort(self, d_in, d_out, d_offsets, arrays, stream=0):
        return check(lib().b200s_sort_ragged(self._h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                                             ctypes.c_void_p(d_offsets), arrays, ctypes.c_void_p(stream)))

    def sort_hinted(self, d_in, d_out, d_offsets, h_offsets_int32, stream=0):
        """sort() with the host copy of the offsets: a plan made with
        PLAN_NO_GRAPH launches only the length classes the batch holds."""
        off = np.ascontiguousarray(h_offsets_int32, dtype=np.int32)
        return check(lib().b200s_sort_ragged_hinted(self._h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                                                    ctypes.c_void_p(d_offsets), ctypes.c_void_p(off.ctypes.data),
                                                    len(off) - 1, ctypes.c_void_p(stream)))

    def too_long(self, stream=0):
        c = ctypes.c_int64(0)
        check(lib().b200s_plan_too_long(self._h, ctypes.c_void_p(stream), ctypes.byref(c)))
        return c.value

    def prepare_plain(self, h_offsets_int32, by_bucket=False):
        """Group the arrays for the plain form: by exact length, or by_bucket by
        power-of-two working length; returns the launches per sort."""
        off = np.ascontiguousarray(h_offsets_int32, dtype=np.int32)
        fn = lib().b200s_plan_prepare_plain_buckets if by_bucket else lib().b200s_plan_prepare_plain
        check(fn(self._h, ctypes.c_void_p(off.ctypes.data), len(off) - 1))
        return lib().b200s_plan_plain_launches(self._h)

    def sort_plain(self, d_in, d_out, d_offsets, stream=0):
        return check(lib().b200s_sort_ragged_plain(self._h, ctypes.c_void_p(d_in), ctypes.c_void_p(d_out),
                                                   ctypes.c_void_p(d_offsets), ctypes.c_void_p(stream)))

    def close(self):
        if self._h:
            lib().b200s_plan_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching sort server (b200s_server_*): submit requests of any
    length as they arrive; the server batches, sorts and returns them."""

    def __init__(self, dtype, budget_bytes=1 << 30, max_inflight=4, max_batch=4096, max_queue=65536, flags=0,
                 device=0):
        self.dtype = dtype
        self._h = ctypes.c_void_p()
        cfg = ServerConfig(device, dtype, flags, budget_bytes, max_inflight, max_batch, max_queue)
        check(lib().b200s_server_create(ctypes.byref(self._h), ctypes.byref(cfg)))

    def submit_status(self, src, dst, n, mem=MEM_DEVICE):
        """Raw status and ticket of one submission (src/dst are integer pointers)."""
        t = ctypes.c_uint64(0)
        st = lib().b200s_server_submit(self._h, ctypes.c_void_p(src), ctypes.c_void_p(dst), n, mem,
                                       ctypes.byref(t))
        return st, t.value

    def submit(self, src, dst, n, mem=MEM_DEVICE):
        st, t = self.submit_status(src, dst, n, mem)
        check(st)
        return t

    def wait(self, ticket, timeout_us=-1):
        """Outcome of a request (a status code), after it finished."""
        r = ctypes.c_int(0)
        check(lib().b200s_server_wait(self._h, ticket, timeout_us, ctypes.byref(r)))
        return r.value

    def poll(self, ticket):
        state, r = ctypes.c_int32(0), ctypes.c_int(0)
        check(lib().b200s_server_poll(self._h, ticket, ctypes.byref(state), ctypes.byref(r)))
        return state.value, r.value

    def cancel(self, ticket):
        return lib().b200s_server_cancel(self._h, ticket)

    def drain(self, timeout_us=-1):
        return check(lib().b200s_server_drain(self._h, timeout_us))

    def stats(self, reset=False):
        s = ServerStats()
        check(lib().b200s_server_stats_get(self._h, ctypes.byref(s), int(reset)))
        return s

    def close(self):
        if self._h:
            lib().b200s_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
