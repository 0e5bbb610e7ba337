"""Python binding of the sort engine's C ABI (include/mgs.h) over ctypes.

The engine itself is native: lib/libmgs.so (CUDA kernels for sm_100a + C++
host runtime). This module only marshals arguments. It never falls back to a
CPU path: if the library or a GPU is missing, calls raise MgsError.

Reference surface (hpides/multi-gpu-sorting) mirrored here:
  TanasicSort<T>(HostVector<T>*, gpus)       -> tanasic_sort(array, gpus)
  GowanlockSort<T>(HostVector<T>*, ...)      -> gowanlock_sort(array, ...)
  DataGenerator(seed).ComputeDistribution<T> -> DataGenerator(seed).compute_distribution(...)
"""
from __future__ import annotations

import ctypes
import os
import weakref

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "lib", "libmgs.so")

MGS_OK = 0
MGS_ERR_INVALID = 1
MGS_ERR_OOM = 2
MGS_ERR_CUDA = 3
MGS_ERR_TIMEOUT = 4
MGS_ERR_NO_DEVICE = 5
MGS_ERR_CANCELLED = 6
MGS_ERR_BUSY = 7

# mgs_dtype codes and their numpy storage types. The reference CLI names
# int/long/float/double (src/sort_benchmark.cu:420-432).
DTYPES = {
    "u32": (0, np.uint32),
    "i32": (1, np.int32),
    "f32": (2, np.float32),
    "u64": (3, np.uint64),
    "i64": (4, np.int64),
    "f64": (5, np.float64),
}
REFERENCE_TYPE_NAMES = {"int": "i32", "long": "i64", "float": "f32", "double": "f64"}
_NP_TO_NAME = {np.dtype(v[1]): k for k, v in DTYPES.items()}


class MgsError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"[mgs status {code}] {message}")
        self.code = code


class ServerConfig(ctypes.Structure):
    _fields_ = [("device", ctypes.c_int), ("num_slots", ctypes.c_int), ("slot_keys", ctypes.c_size_t),
                ("coalesce_keys", ctypes.c_size_t), ("max_batch_requests", ctypes.c_size_t),
                ("device_budget_bytes", ctypes.c_size_t)]


class ServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("rejected", ctypes.c_uint64),
                ("cancelled", ctypes.c_uint64), ("batches", ctypes.c_uint64), ("keys", ctypes.c_uint64),
                ("kernel_launches", ctypes.c_uint64), ("num_slots", ctypes.c_int), ("p50_us", ctypes.c_double),
                ("p99_us", ctypes.c_double), ("mean_us", ctypes.c_double), ("max_us", ctypes.c_double),
                ("busy_s", ctypes.c_double), ("pool_bytes", ctypes.c_uint64), ("pool_free_bytes", ctypes.c_uint64)]


class TuneSample(ctypes.Structure):
    _fields_ = [("key_bytes", ctypes.c_int), ("size_class", ctypes.c_int), ("n", ctypes.c_size_t),
                ("shape", ctypes.c_int), ("rank_mode", ctypes.c_int), ("ms", ctypes.c_double), ("chosen", ctypes.c_int)]


class KernelTime(ctypes.Structure):
    _fields_ = [("name", ctypes.c_char * 48), ("launches", ctypes.c_uint64), ("total_ms", ctypes.c_double)]


_lib = None


def load_library(path: str = LIB_PATH) -> ctypes.CDLL:
    """Loads libmgs.so (once) and declares the C signatures."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise MgsError(MGS_ERR_INVALID, f"engine library not built: {path} (run __graft_entry__.build())")
    lib = ctypes.CDLL(path)
    c_size, c_int, c_void, c_u32 = ctypes.c_size_t, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint32
    sig = {
        "mgs_version": ([], c_int),
        "mgs_last_error_string": ([], ctypes.c_char_p),
        "mgs_dtype_size": ([c_int], c_size),
        "mgs_device_count": ([ctypes.POINTER(c_int)], c_int),
        "mgs_ctx_create": ([c_int, c_size, ctypes.POINTER(c_void)], c_int),
        "mgs_ctx_destroy": ([c_void], c_int),
        "mgs_ctx_synchronize": ([c_void], c_int),
        "mgs_ctx_arena_bytes": ([c_void, ctypes.POINTER(c_size)], c_int),
        "mgs_ctx_set_profiling": ([c_void, c_int], c_int),
        "mgs_ctx_kernel_times": ([c_void, ctypes.POINTER(KernelTime), c_int, ctypes.POINTER(c_int)], c_int),
        "mgs_ctx_launch_count": ([c_void, ctypes.POINTER(ctypes.c_uint64), c_int], c_int),
        "mgs_host_alloc": ([c_size, ctypes.POINTER(c_void)], c_int),
        "mgs_host_free": ([c_void], c_int),
        "mgs_sort_temp_bytes": ([c_int, c_size, ctypes.POINTER(c_size)], c_int),
        "mgs_sort_device": ([c_void, c_int, c_void, c_size, c_void, c_size, c_void], c_int),
        "mgs_sort_host": ([c_void, c_int, c_void, c_size], c_int),
        "mgs_sort_pairs_temp_bytes": ([c_int, c_size, c_size, ctypes.POINTER(c_size)], c_int),
        "mgs_sort_pairs_device": ([c_void, c_int, c_void, c_void, c_size, c_size, c_void, c_size, c_void], c_int),
        "mgs_argsort_device": ([c_void, c_int, c_void, c_void, c_size, c_size, c_void, c_size, c_void], c_int),
        "mgs_sort_range_device": ([c_void, c_int, c_void, c_void, c_size, c_size, c_int, c_int, c_int, c_void, c_size,
                                   c_void], c_int),
        "mgs_sort_device_noalloc": ([c_int, c_void, c_size, c_void], c_int),
        "mgs_generate": ([c_int, ctypes.c_char_p, c_u32, c_void, c_size], c_int),
        "mgs_generate_device": ([c_void, c_int, ctypes.c_char_p, c_u32, c_void, c_size], c_int),
        "mgs_tanasic_sort": ([c_void, c_int, c_void, c_size, c_int], c_int),
        "mgs_tanasic_sort_device": ([c_void, c_int, c_void, c_size, c_int], c_int),
        "mgs_find_pivot_device": ([c_void, c_int, ctypes.POINTER(c_void), ctypes.POINTER(c_void), c_int, c_size,
                                   ctypes.POINTER(c_size)], c_int),
        "mgs_merge_temp_bytes": ([c_int, c_int, c_size, ctypes.POINTER(c_size)], c_int),
        "mgs_merge_device": ([c_void, c_int, c_void, c_size, c_void, c_size, c_void, c_void, c_size, c_void], c_int),
        "mgs_kway_merge_device": ([c_void, c_int, ctypes.POINTER(c_void), ctypes.POINTER(c_size), c_int, c_void,
                                   c_void, c_size, c_void], c_int),
        "mgs_segmented_sort_temp_bytes": ([c_int, c_size, c_size, ctypes.POINTER(c_size)], c_int),
        "mgs_segmented_sort_device": ([c_void, c_int, c_void, c_size, c_void, c_size, c_void, c_size, c_void], c_int),
        "mgs_server_create": ([ctypes.POINTER(ServerConfig), ctypes.POINTER(c_void)], c_int),
        "mgs_server_destroy": ([c_void], c_int),
        "mgs_server_submit": ([c_void, c_int, c_void, c_size, ctypes.POINTER(ctypes.c_uint64)], c_int),
        "mgs_server_submit_device": ([c_void, c_int, c_void, c_size, ctypes.POINTER(ctypes.c_uint64)], c_int),
        "mgs_server_wait": ([c_void, ctypes.c_uint64, c_int, ctypes.POINTER(c_int)], c_int),
        "mgs_server_cancel": ([c_void, ctypes.c_uint64], c_int),
        "mgs_server_stats_get": ([c_void, ctypes.POINTER(ServerStats), c_int], c_int),
        "mgs_gowanlock_sort": ([c_void, c_int, c_void, c_size, c_size, c_size, c_size, c_int], c_int),
        "mgs_ctx_phase_seconds": ([c_void, ctypes.c_char_p, ctypes.POINTER(ctypes.c_double)], c_int),
        "mgs_plan_sort_create": ([c_void, c_int, c_void, c_size, c_void, c_size, ctypes.POINTER(c_void)], c_int),
        "mgs_plan_segmented_create": ([c_void, c_int, c_void, c_size, c_void, c_size, c_void, c_size,
                                       ctypes.POINTER(c_void)], c_int),
        "mgs_plan_launch": ([c_void, c_void], c_int),
        "mgs_plan_launch_count": ([c_void, ctypes.POINTER(ctypes.c_uint64)], c_int),
        "mgs_plan_destroy": ([c_void], c_int),
        "mgs_tune_get": ([c_int, c_size, ctypes.POINTER(c_int), ctypes.POINTER(c_int)], c_int),
        "mgs_tune_set": ([c_int, c_int, c_int, c_int], c_int),
        "mgs_tune_load": ([ctypes.c_char_p], c_int),
        "mgs_tune_save": ([ctypes.c_char_p], c_int),
        "mgs_autotune": ([c_void, c_int, c_size, c_int, ctypes.POINTER(TuneSample), c_int, ctypes.POINTER(c_int)],
                         c_int),
        "mgs_test_set_waits": ([c_int, c_u32, c_u32, c_u32], c_int),
        "mgs_test_fail_device_allocations": ([c_int], c_int),
    }
    for name, (args, res) in sig.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def _check(rc: int) -> None:
    if rc != MGS_OK:
        msg = _lib.mgs_last_error_string()
        raise MgsError(rc, msg.decode() if msg else "")


def dtype_code(dtype) -> int:
    """Accepts 'u32'..'f64', reference names ('int', 'long', ...) or numpy dtypes."""
    if isinstance(dtype, str):
        dtype = REFERENCE_TYPE_NAMES.get(dtype, dtype)
        return DTYPES[dtype][0]
    return DTYPES[_NP_TO_NAME[np.dtype(dtype)]][0]


def np_dtype(dtype) -> np.dtype:
    if isinstance(dtype, str):
        dtype = REFERENCE_TYPE_NAMES.get(dtype, dtype)
        return np.dtype(DTYPES[dtype][1])
    return np.dtype(dtype)


def device_count() -> int:
    lib = load_library()
    c = ctypes.c_int(0)
    rc = lib.mgs_device_count(ctypes.byref(c))
    return c.value if rc == MGS_OK else 0


def host_empty(n: int, dtype) -> np.ndarray:
    """A numpy array backed by pinned host memory (HostVector<T>, src/host_vector.cuh:7)."""
    lib = load_library()
    dt = np_dtype(dtype)
    nbytes = max(int(n) * dt.itemsize, 1)
    p = ctypes.c_void_p()
    _check(lib.mgs_host_alloc(nbytes, ctypes.byref(p)))
    buf = (ctypes.c_char * nbytes).from_address(p.value)
    arr = np.frombuffer(buf, dtype=dt, count=int(n))
    weakref.finalize(buf, lib.mgs_host_free, ctypes.c_void_p(p.value))
    return arr


def generate(dtype, distribution: str, seed: int, n: int, out: np.ndarray | None = None) -> np.ndarray:
    """DataGenerator(seed).ComputeDistribution<T>(out, n, distribution) (src/data_generator.cuh:18-36)."""
    lib = load_library()
    dt = np_dtype(dtype)
    if out is None:
        out = np.zeros(int(n), dtype=dt)
    assert out.dtype == dt and out.flags.c_contiguous and out.size >= n
    _check(lib.mgs_generate(dtype_code(dtype), distribution.encode(), int(seed) & 0xFFFFFFFF,
                            out.ctypes.data_as(ctypes.c_void_p), int(n)))
    return out


def tune_get(dtype, n: int) -> tuple:
    """(shape, rank_mode) the radix sort uses for n keys of this dtype (mgs_tune_get)."""
    lib = load_library()
    shape, mode = ctypes.c_int(), ctypes.c_int()
    _check(lib.mgs_tune_get(dtype_code(dtype), int(n), ctypes.byref(shape), ctypes.byref(mode)))
    return shape.value, mode.value


def tune_set(dtype, size_class: int, shape: int, rank_mode: int) -> None:
    lib = load_library()
    _check(lib.mgs_tune_set(dtype_code(dtype), int(size_class), int(shape), int(rank_mode)))


def tune_load(path: str) -> None:
    lib = load_library()
    _check(lib.mgs_tune_load(path.encode()))


def tune_save(path: str) -> None:
    lib = load_library()
    _check(lib.mgs_tune_save(path.encode()))


def sort_device_noalloc(d_keys: int, n: int, dtype, stream: int = 0) -> None:
    """mgs_sort_device_noalloc: the device sort without any allocation (fixed 32 MiB scratch in
    the library's device image; at most 2^22 4-byte or 2^21 8-byte keys). For callers
    that cannot call cudaMalloc. Calls that overlap on one GPU race."""
    lib = load_library()
    _check(lib.mgs_sort_device_noalloc(dtype_code(dtype), ctypes.c_void_p(d_keys), int(n),
                                       ctypes.c_void_p(stream or None)))


NO_HELD_TILE = 0xFFFFFFFF


def inject_waits(device: int = 0, lookback_spins: int = 0, tma_polls: int = 0, hold_tile: int = NO_HELD_TILE):
    """mgs_test_set_waits (failure injection for tests): bounds of the device-side waits (0 = default) and a
    tile of the plain device sort whose look-back status is never published. Defaults restore normal sorts."""
    _check(load_library().mgs_test_set_waits(int(device), int(lookback_spins), int(tma_polls), int(hold_tile)))


def inject_allocation_failures(count: int) -> None:
    """mgs_test_fail_device_allocations (failure injection for tests): the next `count` arena growths fail
    with MGS_ERR_OOM."""
    _check(load_library().mgs_test_fail_device_allocations(int(count)))


class DataGenerator:
    """Mirror of the reference's DataGenerator (src/data_generator.cuh:12-211)."""

    def __init__(self, distribution_seed: int):
        self.distribution_seed = int(distribution_seed) & 0xFFFFFFFF

    def compute_distribution(self, begin: np.ndarray, num_elements: int, distribution_type: str) -> None:
        generate(begin.dtype, distribution_type, self.distribution_seed, num_elements, out=begin)


class Plan:
    """A recorded sort (mgs_plan): launch() replays it on a stream; close() waits for the device and frees it.
    The context that made it must stay open while the plan lives."""

    def __init__(self, ctx: "Context", handle: ctypes.c_void_p):
        self.ctx = ctx
        self._lib = ctx._lib
        self.handle = handle

    def launch(self, stream: int = 0) -> None:
        _check(self._lib.mgs_plan_launch(self.handle, ctypes.c_void_p(stream or None)))

    def launch_count(self) -> int:
        v = ctypes.c_uint64()
        _check(self._lib.mgs_plan_launch_count(self.handle, ctypes.byref(v)))
        return int(v.value)

    def close(self) -> None:
        """Frees the plan; a plan whose context was already closed is dropped without touching the context."""
        if self.handle:
            h, self.handle = self.handle, None
            if self.ctx._fin.alive:
                _check(self._lib.mgs_plan_destroy(h))

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Context:
    """One engine context per device (streams, device arena, status word)."""

    def __init__(self, device: int = 0, arena_bytes: int = 0):
        self._lib = load_library()
        h = ctypes.c_void_p()
        _check(self._lib.mgs_ctx_create(int(device), int(arena_bytes), ctypes.byref(h)))
        self.handle = h
        self.device = device
        self._fin = weakref.finalize(self, self._lib.mgs_ctx_destroy, h)

    def close(self) -> None:
        if self._fin.alive:
            self._fin()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # --- device-resident sort (thrust::sort on one GPU) ---
    @staticmethod
    def sort_temp_bytes(dtype, n: int) -> int:
        lib = load_library()
        b = ctypes.c_size_t()
        _check(lib.mgs_sort_temp_bytes(dtype_code(dtype), int(n), ctypes.byref(b)))
        return b.value

    def sort_device(self, d_keys: int, n: int, dtype, d_temp: int = 0, temp_bytes: int = 0,
                    stream: int = 0) -> None:
        _check(self._lib.mgs_sort_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys), int(n),
                                         ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                         ctypes.c_void_p(stream or None)))

    # --- key-value sort and argsort (thrust::sort_by_key order) ---
    @staticmethod
    def sort_pairs_temp_bytes(dtype, value_bytes: int, n: int) -> int:
        lib = load_library()
        b = ctypes.c_size_t()
        _check(lib.mgs_sort_pairs_temp_bytes(dtype_code(dtype), int(value_bytes), int(n), ctypes.byref(b)))
        return b.value

    def sort_pairs_device(self, d_keys: int, d_values: int, value_bytes: int, n: int, dtype, d_temp: int = 0,
                          temp_bytes: int = 0, stream: int = 0) -> None:
        _check(self._lib.mgs_sort_pairs_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys),
                                               ctypes.c_void_p(d_values), int(value_bytes), int(n),
                                               ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                               ctypes.c_void_p(stream or None)))

    def argsort_device(self, d_keys: int, d_indices: int, index_bytes: int, n: int, dtype, d_temp: int = 0,
                       temp_bytes: int = 0, stream: int = 0) -> None:
        _check(self._lib.mgs_argsort_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys),
                                            ctypes.c_void_p(d_indices), int(index_bytes), int(n),
                                            ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                            ctypes.c_void_p(stream or None)))

    def sort_range_device(self, d_keys: int, n: int, dtype, begin_bit: int, end_bit: int, descending: bool = False,
                          d_values: int = 0, value_bytes: int = 0, d_temp: int = 0, temp_bytes: int = 0,
                          stream: int = 0) -> None:
        """Sort by bits [begin_bit, end_bit) of the ordered keys, ascending or descending (mgs_sort_range_device)."""
        _check(self._lib.mgs_sort_range_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys),
                                               ctypes.c_void_p(d_values or None), int(value_bytes), int(n),
                                               int(begin_bit), int(end_bit), 1 if descending else 0,
                                               ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                               ctypes.c_void_p(stream or None)))

    def generate_device(self, d_out: int, n: int, dtype, distribution: str, seed: int) -> None:
        """The bytes of generate(dtype, distribution, seed, n), written straight into device memory
        (mgs_generate_device); refuses the distributions that use the host's log/cos."""
        _check(self._lib.mgs_generate_device(self.handle, dtype_code(dtype), distribution.encode(),
                                             int(seed) & 0xFFFFFFFF, ctypes.c_void_p(d_out or None), int(n)))

    # --- TanasicSort with one GPU: host buffer in, sorted in place ---
    def sort_host(self, keys: np.ndarray) -> None:
        assert keys.flags.c_contiguous
        _check(self._lib.mgs_sort_host(self.handle, dtype_code(keys.dtype), keys.ctypes.data_as(ctypes.c_void_p),
                                       keys.size))

    # --- TanasicSort with g partitions as chunks of this GPU ---
    def tanasic_sort(self, keys: np.ndarray, num_chunks: int = 1) -> None:
        """TanasicSort<T>(&keys, gpus) with len(gpus) == num_chunks (src/tanasic_sort.cuh:223-299)."""
        assert keys.flags.c_contiguous
        _check(self._lib.mgs_tanasic_sort(self.handle, dtype_code(keys.dtype), keys.ctypes.data_as(ctypes.c_void_p),
                                          keys.size, int(num_chunks)))

    def tanasic_sort_device(self, d_keys: int, n: int, dtype, num_chunks: int) -> None:
        _check(self._lib.mgs_tanasic_sort_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys), int(n),
                                                 int(num_chunks)))

    def find_pivot_device(self, left: list, right: list, chunk_size: int, dtype) -> int:
        half = len(left)
        lp = (ctypes.c_void_p * half)(*left)
        rp = (ctypes.c_void_p * half)(*right)
        out = ctypes.c_size_t()
        _check(self._lib.mgs_find_pivot_device(self.handle, dtype_code(dtype), lp, rp, half, int(chunk_size),
                                               ctypes.byref(out)))
        return out.value

    @staticmethod
    def merge_temp_bytes(dtype, k: int, total: int) -> int:
        lib = load_library()
        b = ctypes.c_size_t()
        _check(lib.mgs_merge_temp_bytes(dtype_code(dtype), int(k), int(total), ctypes.byref(b)))
        return b.value

    def merge_device(self, d_a: int, na: int, d_b: int, nb: int, d_out: int, dtype, d_temp: int = 0,
                     temp_bytes: int = 0, stream: int = 0) -> None:
        _check(self._lib.mgs_merge_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_a), int(na),
                                          ctypes.c_void_p(d_b), int(nb), ctypes.c_void_p(d_out),
                                          ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                          ctypes.c_void_p(stream or None)))

    def kway_merge_device(self, d_runs: list, lens: list, d_out: int, dtype, d_temp: int = 0, temp_bytes: int = 0,
                          stream: int = 0) -> None:
        k = len(d_runs)
        rp = (ctypes.c_void_p * k)(*[p or None for p in d_runs])
        lp = (ctypes.c_size_t * k)(*[int(x) for x in lens])
        _check(self._lib.mgs_kway_merge_device(self.handle, dtype_code(dtype), rp, lp, k, ctypes.c_void_p(d_out),
                                               ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                               ctypes.c_void_p(stream or None)))

    # --- batched segmented sort ---
    @staticmethod
    def segmented_sort_temp_bytes(dtype, n: int, num_segments: int) -> int:
        lib = load_library()
        b = ctypes.c_size_t()
        _check(lib.mgs_segmented_sort_temp_bytes(dtype_code(dtype), int(n), int(num_segments), ctypes.byref(b)))
        return b.value

    def segmented_sort_device(self, d_keys: int, n: int, d_offsets: int, num_segments: int, dtype, d_temp: int = 0,
                              temp_bytes: int = 0, stream: int = 0) -> None:
        _check(self._lib.mgs_segmented_sort_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys), int(n),
                                                   ctypes.c_void_p(d_offsets), int(num_segments),
                                                   ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                                   ctypes.c_void_p(stream or None)))

    # --- autotuner ---
    def autotune(self, dtype, max_n: int, reps: int = 3) -> list:
        """Times every onesweep variant per size class up to max_n and keeps the fastest (mgs_autotune)."""
        cap = 256
        arr = (TuneSample * cap)()
        cnt = ctypes.c_int()
        _check(self._lib.mgs_autotune(self.handle, dtype_code(dtype), int(max_n), int(reps), arr, cap,
                                      ctypes.byref(cnt)))
        return [{f: getattr(arr[i], f) for f, _ in TuneSample._fields_} for i in range(min(cnt.value, cap))]

    # --- recorded sorts (CUDA graphs) ---
    def plan_sort(self, d_keys: int, n: int, dtype, d_temp: int = 0, temp_bytes: int = 0) -> "Plan":
        """Records the device sort of the fixed buffer d_keys[0..n) into a CUDA graph (mgs_plan_sort_create)."""
        h = ctypes.c_void_p()
        _check(self._lib.mgs_plan_sort_create(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys), int(n),
                                              ctypes.c_void_p(d_temp or None), int(temp_bytes), ctypes.byref(h)))
        return Plan(self, h)

    def plan_segmented(self, d_keys: int, n: int, d_offsets: int, num_segments: int, dtype, d_temp: int = 0,
                       temp_bytes: int = 0) -> "Plan":
        """Records the segmented sort of fixed buffers into a CUDA graph (mgs_plan_segmented_create)."""
        h = ctypes.c_void_p()
        _check(self._lib.mgs_plan_segmented_create(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys), int(n),
                                                   ctypes.c_void_p(d_offsets), int(num_segments),
                                                   ctypes.c_void_p(d_temp or None), int(temp_bytes),
                                                   ctypes.byref(h)))
        return Plan(self, h)

    # --- GowanlockSort with one GPU: out-of-core chunk pipeline ---
    def gowanlock_sort(self, keys: np.ndarray, chunk_size: int = 0, merge_group_size: int = 0, num_buffers: int = 2,
                       merge_on_gpu: bool = True) -> None:
        """GowanlockSort<T>(&keys, chunk_size, merge_group_size, num_buffers, gpus) (src/gowanlock_sort.cuh:395)."""
        assert keys.flags.c_contiguous
        _check(self._lib.mgs_gowanlock_sort(self.handle, dtype_code(keys.dtype), keys.ctypes.data_as(ctypes.c_void_p),
                                            keys.size, int(chunk_size), int(merge_group_size), int(num_buffers),
                                            0 if merge_on_gpu else 1))

    def phase_seconds(self, phase: str) -> float:
        v = ctypes.c_double()
        _check(self._lib.mgs_ctx_phase_seconds(self.handle, phase.encode(), ctypes.byref(v)))
        return v.value

    def synchronize(self) -> None:
        _check(self._lib.mgs_ctx_synchronize(self.handle))

    def arena_bytes(self) -> int:
        b = ctypes.c_size_t()
        _check(self._lib.mgs_ctx_arena_bytes(self.handle, ctypes.byref(b)))
        return b.value

    def set_profiling(self, enabled: bool) -> None:
        _check(self._lib.mgs_ctx_set_profiling(self.handle, 1 if enabled else 0))

    def kernel_times(self) -> dict:
        cap = 64
        arr = (KernelTime * cap)()
        cnt = ctypes.c_int()
        _check(self._lib.mgs_ctx_kernel_times(self.handle, arr, cap, ctypes.byref(cnt)))
        return {arr[i].name.decode(): (int(arr[i].launches), float(arr[i].total_ms)) for i in range(min(cnt.value, cap))}

    def launch_count(self, reset: bool = False) -> int:
        v = ctypes.c_uint64()
        _check(self._lib.mgs_ctx_launch_count(self.handle, ctypes.byref(v), 1 if reset else 0))
        return int(v.value)


class Server:
    """The serving loop (mgs_server_*): continuous batching of sort requests on one GPU."""

    def __init__(self, device: int = 0, num_slots: int = 4, slot_keys: int = 0, coalesce_keys: int = 1 << 20,
                 max_batch_requests: int = 0, device_budget_bytes: int = 0):
        self._lib = load_library()
        cfg = ServerConfig(device, num_slots, slot_keys, coalesce_keys, max_batch_requests, device_budget_bytes)
        h = ctypes.c_void_p()
        _check(self._lib.mgs_server_create(ctypes.byref(cfg), ctypes.byref(h)))
        self.handle = h
        self._keep = {}
        self._fin = weakref.finalize(self, self._lib.mgs_server_destroy, h)

    def close(self) -> None:
        if self._fin.alive:
            self._fin()

    def submit(self, keys: np.ndarray) -> int:
        """Queues keys (sorted in place); returns the request id. Keep `keys` alive until wait()."""
        assert keys.flags.c_contiguous
        rid = ctypes.c_uint64()
        _check(self._lib.mgs_server_submit(self.handle, dtype_code(keys.dtype), keys.ctypes.data_as(ctypes.c_void_p),
                                           keys.size, ctypes.byref(rid)))
        self._keep[rid.value] = keys
        return rid.value

    def submit_device(self, d_keys: int, n: int, dtype, keep=None) -> int:
        """Queues n keys of `dtype` at device address d_keys (this server's GPU), sorted in place; returns the
        request id. The buffer must stay valid until wait(); `keep` is held until then (e.g. the tensor)."""
        rid = ctypes.c_uint64()
        _check(self._lib.mgs_server_submit_device(self.handle, dtype_code(dtype), ctypes.c_void_p(d_keys), int(n),
                                                  ctypes.byref(rid)))
        self._keep[rid.value] = keep
        return rid.value

    def wait(self, request_id: int, timeout_ms: int = -1) -> int:
        st = ctypes.c_int()
        _check(self._lib.mgs_server_wait(self.handle, request_id, timeout_ms, ctypes.byref(st)))
        self._keep.pop(request_id, None)
        return st.value

    def cancel(self, request_id: int) -> None:
        _check(self._lib.mgs_server_cancel(self.handle, request_id))

    def stats(self, reset: bool = False) -> dict:
        st = ServerStats()
        _check(self._lib.mgs_server_stats_get(self.handle, ctypes.byref(st), 1 if reset else 0))
        return {name: getattr(st, name) for name, _ in ServerStats._fields_}
