"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE).

Used only by tests/, by the smoke entry and by the CPU-baseline and
reference legs of bench.py, always as the checker or as the timed CPU
baseline, never as the product path.  The libraries it loads are built by
oracle/Makefile: _build/liboracle.so (the CPU restatement in oracle.cpp) and,
when the reference was available at build time, _ref/libref_cpu.so and
_ref/libref_gpu_{int,rec}.so (the reference's own code compiled from its headers).
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_CPU_LIB = os.path.join(HERE, "_ref", "libref_cpu.so")
REF_GPU_LIBS = {"int": os.path.join(HERE, "_ref", "libref_gpu_int.so"),
                "rec": os.path.join(HERE, "_ref", "libref_gpu_rec.so")}

MODE_STD, MODE_NETWORK, MODE_STABLE = 0, 1, 2

# reference distributions (valgen.hpp:7-15, bench.cu:26-31)
REF_DISTRIBUTIONS = {"SORTED": 0, "REVERSED": 1, "RANDOM": 2, "NORMAL": 3, "CONSTANT": 4, "BINARY": 5,
                     "PERTURBED_2": 6, "PERTURBED_8": 7, "PERTURBED_32": 8, "EXTREMES": 9}

_orc = None
_ref_cpu = None
_ref_gpu = None


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data)


def lib():
    global _orc
    if _orc is None:
        if not os.path.exists(ORACLE_LIB):
            raise ImportError("oracle not built: run `make -C oracle`")
        h = ctypes.CDLL(ORACLE_LIB)
        h.orc_sort_packed.restype = ctypes.c_int
        h.orc_sort_packed.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int64,
                                      ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        h.orc_sort_ragged.restype = ctypes.c_int
        h.orc_sort_ragged.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_int64, ctypes.c_int, ctypes.c_int]
        h.orc_validate_records.restype = ctypes.c_int64
        h.orc_validate_records.argtypes = [ctypes.c_void_p] * 4 + [ctypes.c_int64]
        h.orc_mix_bits.restype = ctypes.c_uint32
        h.orc_mix_bits.argtypes = [ctypes.c_uint32]
        h.orc_ref_initialize.restype = ctypes.c_int
        h.orc_ref_initialize.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_int64, ctypes.c_int64,
                                         ctypes.c_int]
        _orc = h
    return _orc


def sort_packed(dtype, data, n, arrays, mode=MODE_STD, threads=1):
    """Per-array sort of a packed batch; returns a new array."""
    data = np.ascontiguousarray(data)
    out = np.empty_like(data)
    if lib().orc_sort_packed(dtype, _ptr(data), _ptr(out), n, arrays, mode, threads) != 0:
        raise ValueError("orc_sort_packed rejected its arguments")
    return out


def sort_ragged(dtype, data, offsets, mode=MODE_STD, threads=1):
    data = np.ascontiguousarray(data)
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    out = data.copy()
    if lib().orc_sort_ragged(dtype, _ptr(data), _ptr(out), _ptr(off), len(off) - 1, mode, threads) != 0:
        raise ValueError("orc_sort_ragged rejected its arguments")
    return out


def validate_records(inp, result, expected, offsets):
    """Failing output positions under the reference's record validation."""
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    return int(lib().orc_validate_records(_ptr(inp), _ptr(result), _ptr(expected), _ptr(off), len(off) - 1))


def mix_bits(x):
    return int(lib().orc_mix_bits(x & 0xFFFFFFFF))


def ref_initialize(dtype, n, arrays, distribution, np_dtype):
    """The reference's own batch initialiser (bench.cu:159-192), dtype 0 or 1."""
    out = np.empty(n * arrays, dtype=np_dtype)
    if lib().orc_ref_initialize(dtype, _ptr(out), n, arrays, REF_DISTRIBUTIONS[distribution]) != 0:
        raise ValueError("orc_ref_initialize rejected its arguments")
    return out


# ---- the reference's own code (built from its headers) -------------------------

def ref_cpu_available():
    return os.path.exists(REF_CPU_LIB)


def ref_cpu():
    global _ref_cpu
    if _ref_cpu is None:
        h = ctypes.CDLL(REF_CPU_LIB)
        h.ref_cpu_sort.restype = ctypes.c_int
        h.ref_cpu_sort.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_longlong, ctypes.c_longlong,
                                   ctypes.c_int]
        h.ref_cpu_sort_ragged.restype = ctypes.c_int
        h.ref_cpu_sort_ragged.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_longlong,
                                          ctypes.c_int]
        _ref_cpu = h
    return _ref_cpu


def ref_cpu_sort_inplace(type_code, data, n, arrays, threads):
    """The reference's per-array std::sort (bench.cu:300-301), in place."""
    if ref_cpu().ref_cpu_sort(type_code, _ptr(data), n, arrays, threads) != 0:
        raise ValueError("ref_cpu_sort rejected its arguments")


def ref_cpu_sort_ragged_inplace(type_code, data, offsets, threads):
    """The reference's std::sort applied to every array of a CSR batch, in place."""
    off = np.ascontiguousarray(offsets, dtype=np.int64)
    if ref_cpu().ref_cpu_sort_ragged(type_code, _ptr(data), _ptr(off), len(off) - 1, threads) != 0:
        raise ValueError("ref_cpu_sort_ragged rejected its arguments")


def ref_gpu_available():
    return all(os.path.exists(p) for p in REF_GPU_LIBS.values())


def ref_gpu(suffix):
    """Reference GPU kernels ref_{v6,v3,v4,v12,warp,partition_v3}_<suffix>, suffix "int" or "rec"."""
    global _ref_gpu
    if _ref_gpu is None:
        _ref_gpu = {}
    if suffix not in _ref_gpu:
        h = ctypes.CDLL(REF_GPU_LIBS[suffix])
        for name in ("ref_v6", "ref_v3", "ref_v4"):
            fn = getattr(h, "%s_%s" % (name, suffix))
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                           ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        fn = getattr(h, "ref_warp_%s" % suffix)
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p]
        fn = getattr(h, "ref_v12_%s" % suffix)
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_void_p] + [ctypes.c_int] * 6 + [ctypes.c_void_p]
        fn = getattr(h, "ref_partition_v3_%s" % suffix)
        fn.restype = ctypes.c_int
        fn.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                       ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), ctypes.c_void_p]
        _ref_gpu[suffix] = h
    return _ref_gpu[suffix]
