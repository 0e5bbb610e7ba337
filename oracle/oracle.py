"""ORACLE — test infrastructure only. Not part of the product.

ctypes access to the CPU restatement (_build/liboracle.so, oracle.cpp) and to
the reference's own code compiled from its sources (_ref/libref.so,
ref_wrap.cu). Only tests/, __graft_entry__.smoke() and bench.py's CPU
baseline legs import this module, and only to check or to time the
reference; the engine never calls it.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libref.so")

DTYPE_CODES = {np.dtype(np.uint32): 0, np.dtype(np.int32): 1, np.dtype(np.float32): 2,
               np.dtype(np.uint64): 3, np.dtype(np.int64): 4, np.dtype(np.float64): 5}

_oracle = None
_ref = None


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(ctypes.c_void_p)


def oracle_lib() -> ctypes.CDLL:
    global _oracle
    if _oracle is None:
        lib = ctypes.CDLL(ORACLE_LIB)
        v, s, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        lib.oracle_sort.argtypes = [i, v, s]
        lib.oracle_merge.argtypes = [i, v, s, v, s, v]
        lib.oracle_find_pivot.argtypes = [i, v, s, i, ctypes.POINTER(s)]
        lib.oracle_tanasic_sort.argtypes = [i, v, s, i]
        lib.oracle_kway_merge.argtypes = [i, ctypes.POINTER(v), ctypes.POINTER(s), i, v]
        lib.oracle_segmented_sort.argtypes = [i, v, ctypes.POINTER(ctypes.c_uint64), s]
        lib.oracle_sort_pairs.argtypes = [i, v, v, s, s]
        lib.oracle_sort_range.argtypes = [i, v, v, s, s, i, i, i]
        lib.oracle_order_key.argtypes = [i, ctypes.c_uint64]
        lib.oracle_order_key.restype = ctypes.c_uint64
        _oracle = lib
    return _oracle


def ref_available() -> bool:
    return os.path.exists(REF_LIB)


def ref_lib() -> ctypes.CDLL:
    global _ref
    if _ref is None:
        lib = ctypes.CDLL(REF_LIB)
        v, s, i = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int
        lib.ref_generate.argtypes = [i, ctypes.c_char_p, ctypes.c_uint32, v, s]
        lib.ref_tanasic_sort.argtypes = [i, v, s, i]
        lib.ref_gowanlock_sort.argtypes = [i, v, s, s, s, s, i, i]
        lib.ref_gnu_parallel_sort.argtypes = [i, v, s, i]
        lib.ref_multiway_merge.argtypes = [i, ctypes.POINTER(v), ctypes.POINTER(s), i, v, i]
        lib.ref_phase_seconds.argtypes = [ctypes.c_char_p]
        lib.ref_phase_seconds.restype = ctypes.c_double
        lib.ref_num_procs.restype = i
        lib.ref_cub_sort_device_ms.argtypes = [i, v, v, s, v, s, ctypes.POINTER(s)]
        lib.ref_cub_sort_device_ms.restype = ctypes.c_double
        lib.ref_thrust_sort_by_key.argtypes = [i, v, v, s, s]
        lib.ref_cub_sort_range.argtypes = [i, v, v, s, s, i, i, i]
        _ref = lib
    return _ref


def code(a: np.ndarray) -> int:
    return DTYPE_CODES[a.dtype]


# ---- restatement -------------------------------------------------------------
def sort(a: np.ndarray) -> np.ndarray:
    """thrust::sort order (CUB 2.8.2 radix order, stable); returns a sorted copy."""
    out = np.ascontiguousarray(a).copy()
    assert oracle_lib().oracle_sort(code(out), _ptr(out), out.size) == 0
    return out


def sort_pairs(keys: np.ndarray, values: np.ndarray):
    """thrust::sort_by_key order: keys sorted as by sort(), values following their keys, equal keys in input
    order. Returns sorted copies (keys, values); values are 4- or 8-byte payloads."""
    k = np.ascontiguousarray(keys).copy()
    v = np.ascontiguousarray(values).copy()
    assert k.size == v.size
    assert oracle_lib().oracle_sort_pairs(code(k), _ptr(k), _ptr(v), v.dtype.itemsize, k.size) == 0
    return k, v


def sort_range(keys: np.ndarray, begin_bit: int, end_bit: int, descending: bool = False, values=None):
    """CUB begin_bit / end_bit (and descending) order: stable sort by bits [begin_bit, end_bit) of the ordered
    keys. Returns sorted copies: keys, or (keys, values) when values are given."""
    k = np.ascontiguousarray(keys).copy()
    v = None if values is None else np.ascontiguousarray(values).copy()
    vb = 0 if v is None else v.dtype.itemsize
    assert oracle_lib().oracle_sort_range(code(k), _ptr(k), None if v is None else _ptr(v), vb, k.size, begin_bit,
                                          end_bit, 1 if descending else 0) == 0
    return k if v is None else (k, v)


def merge(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    out = np.empty(a.size + b.size, dtype=a.dtype)
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert oracle_lib().oracle_merge(code(a), _ptr(a), a.size, _ptr(b), b.size, _ptr(out)) == 0
    return out


def find_pivot(parts: np.ndarray, psize: int, g: int) -> int:
    p = ctypes.c_size_t()
    parts = np.ascontiguousarray(parts)
    assert oracle_lib().oracle_find_pivot(code(parts), _ptr(parts), psize, g, ctypes.byref(p)) == 0
    return p.value


def tanasic_sort(a: np.ndarray, g: int) -> np.ndarray:
    out = np.ascontiguousarray(a).copy()
    assert oracle_lib().oracle_tanasic_sort(code(out), _ptr(out), out.size, g) == 0
    return out


def kway_merge(runs: list) -> np.ndarray:
    runs = [np.ascontiguousarray(r) for r in runs]
    total = sum(r.size for r in runs)
    dt = runs[0].dtype
    out = np.empty(total, dtype=dt)
    ptrs = (ctypes.c_void_p * len(runs))(*[r.ctypes.data for r in runs])
    lens = (ctypes.c_size_t * len(runs))(*[r.size for r in runs])
    assert oracle_lib().oracle_kway_merge(DTYPE_CODES[dt], ptrs, lens, len(runs), _ptr(out)) == 0
    return out


def segmented_sort(a: np.ndarray, offsets: np.ndarray) -> np.ndarray:
    out = np.ascontiguousarray(a).copy()
    offs = np.ascontiguousarray(offsets, dtype=np.uint64)
    assert oracle_lib().oracle_segmented_sort(code(out), _ptr(out),
                                              offs.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)),
                                              offs.size - 1) == 0
    return out


def order_keys(a: np.ndarray) -> np.ndarray:
    """Radix-order keys (unsigned) of every element, vectorised in numpy."""
    bits = a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)
    ut = bits.dtype.type
    sign = ut(1) << ut(bits.dtype.itemsize * 8 - 1)
    if a.dtype.kind == "u":
        return bits.copy()
    if a.dtype.kind == "i":
        return bits ^ sign
    b = np.where(bits == sign, ut(0), bits)
    return np.where(b & sign, ~b, b ^ sign)


# ---- the reference's own code --------------------------------------------------
def ref_generate(dtype, distribution: str, seed: int, n: int) -> np.ndarray:
    out = np.zeros(n, dtype=dtype)
    assert ref_lib().ref_generate(code(out), distribution.encode(), seed & 0xFFFFFFFF, _ptr(out), n) == 0
    return out


def ref_gnu_parallel_sort(a: np.ndarray, threads: int) -> np.ndarray:
    """Sorts `a` in place with the reference's gnu_parallel branch; returns seconds (sort_phase)."""
    assert ref_lib().ref_gnu_parallel_sort(code(a), _ptr(a), a.size, int(threads)) == 0
    return ref_lib().ref_phase_seconds(b"sort_phase")


def ref_multiway_merge(runs: list, threads: int):
    runs = [np.ascontiguousarray(r) for r in runs]
    total = sum(r.size for r in runs)
    dt = runs[0].dtype
    out = np.empty(total, dtype=dt)
    ptrs = (ctypes.c_void_p * len(runs))(*[r.ctypes.data for r in runs])
    lens = (ctypes.c_size_t * len(runs))(*[r.size for r in runs])
    assert ref_lib().ref_multiway_merge(DTYPE_CODES[dt], ptrs, lens, len(runs), _ptr(out), int(threads)) == 0
    return out, ref_lib().ref_phase_seconds(b"merge_phase")


def ref_tanasic_sort(a: np.ndarray, device: int = 0) -> None:
    """The reference's TanasicSort<T> with one GPU (runs thrust::sort on the device), in place."""
    assert ref_lib().ref_tanasic_sort(code(a), _ptr(a), a.size, device) == 0


def ref_gowanlock_sort(a: np.ndarray, chunk_size: int = 0, merge_group_size: int = 0, num_buffers: int = 2,
                       device: int = 0, threads: int = 8) -> None:
    assert ref_lib().ref_gowanlock_sort(code(a), _ptr(a), a.size, chunk_size, merge_group_size, num_buffers,
                                        device, threads) == 0


def ref_cub_sort_device_ms(dtype_code: int, d_keys_in: int, d_keys_out: int, n: int, d_temp: int = 0,
                           temp_bytes: int = 0):
    """cub::DeviceRadixSort::SortKeys from device keys d_keys_in into d_keys_out (out of place, as CUB requires;
    src/local_gpu_sort_algorithm_benchmark.cu:51-67). Returns (ms, temp bytes CUB needs); ms < 0 when only the
    size was queried."""
    need = ctypes.c_size_t()
    ms = ref_lib().ref_cub_sort_device_ms(dtype_code, ctypes.c_void_p(d_keys_in or None),
                                          ctypes.c_void_p(d_keys_out or None), n, ctypes.c_void_p(d_temp or None),
                                          temp_bytes, ctypes.byref(need))
    return ms, need.value


def ref_cub_sort(dtype_code: int, d_keys: int, n: int, w: int) -> None:
    """The reference's sort order on device keys, in place: cub::DeviceRadixSort::SortKeys over all 8*w bits
    (the library thrust::sort dispatches to, src/tanasic_sort.cuh:264), run out of place and copied back."""
    ref_cub_sort_range(dtype_code, d_keys, n, 0, 8 * w, False)


def ref_thrust_sort_by_key(dtype_code: int, d_keys: int, d_values: int, value_bytes: int, n: int) -> None:
    """thrust::sort_by_key on device keys (of the given dtype code) and 4- or 8-byte values, in place."""
    assert ref_lib().ref_thrust_sort_by_key(dtype_code, ctypes.c_void_p(d_keys), ctypes.c_void_p(d_values),
                                            value_bytes, n) == 0


def ref_cub_sort_range(dtype_code: int, d_keys: int, n: int, begin_bit: int, end_bit: int, descending: bool,
                       d_values: int = 0, value_bytes: int = 0) -> None:
    """cub::DeviceRadixSort::SortKeys/SortPairs[Descending] with begin_bit / end_bit, in place on device buffers."""
    assert ref_lib().ref_cub_sort_range(dtype_code, ctypes.c_void_p(d_keys), ctypes.c_void_p(d_values or None),
                                        value_bytes, n, begin_bit, end_bit, 1 if descending else 0) == 0


def ref_num_procs() -> int:
    return ref_lib().ref_num_procs()


def ref_phase_seconds(phase: str) -> float:
    """The reference's TimeDurations entry `phase` (src/time_durations.cuh) of its last timed call, in seconds."""
    return ref_lib().ref_phase_seconds(phase.encode())
