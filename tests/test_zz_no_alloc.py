"""The allocation-free sort entry point, mgs_sort_device_noalloc.

It exists for callers that cannot allocate device memory (code running while a
pool or arena owns the device memory, allocators that must not re-enter
cudaMalloc, servers that forbid allocation after start-up). It sorts with a
fixed scratch area in the library's device image, so it must give exactly the
output of the allocating entry point, mgs_sort_device, call after call: the
scratch keeps the previous call's contents and each call must clear what has
to start at zero. This file runs last so that a failure here leaves every other
test already run; it also passes on its own in a fresh process.
"""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

MAX_KEYS = {4: 1 << 22, 8: 1 << 21}


def noalloc_fn(mgs):
    lib = mgs.load_library()
    fn = lib.mgs_sort_device_noalloc
    fn.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    return lib, fn


def on_device(a):
    st = np.int32 if a.dtype.itemsize == 4 else np.int64
    return torch.from_numpy(a.view(st).copy()).cuda()


@pytest.mark.parametrize("dtype,dist,n", [
    ("u32", "uniform", 1_000_003),
    ("u64", "uniform", 1 << 21),
    ("f32", "full-uniform-specials", 777_777),
    ("u64", "full-uniform", 500_001),
    ("i32", "zipf", 65_537),
])
def test_noalloc_matches_sort_device_on_two_calls_in_a_row(ctx, mgs, dtype, dist, n):
    lib, fn = noalloc_fn(mgs)
    code = mgs.dtype_code(dtype)
    for call in range(2):
        a = mgs.generate(dtype, dist, 100 + call, n)
        want = on_device(a)
        got = on_device(a)
        torch.cuda.synchronize()
        ctx.sort_device(want.data_ptr(), n, dtype)
        ctx.synchronize()
        stream = torch.cuda.current_stream().cuda_stream
        assert fn(code, ctypes.c_void_p(got.data_ptr()), n, ctypes.c_void_p(stream)) == mgs.MGS_OK, \
            lib.mgs_last_error_string()
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"call {call}: noalloc sort differs from mgs_sort_device"


def test_noalloc_largest_and_oversized_inputs(ctx, mgs):
    lib, fn = noalloc_fn(mgs)
    n = MAX_KEYS[4]
    a = mgs.generate("u32", "uniform", 5, n)
    want = on_device(a)
    got = on_device(a)
    torch.cuda.synchronize()
    ctx.sort_device(want.data_ptr(), n, "u32")
    ctx.synchronize()
    stream = torch.cuda.current_stream().cuda_stream
    assert fn(0, ctypes.c_void_p(got.data_ptr()), n, ctypes.c_void_p(stream)) == mgs.MGS_OK
    torch.cuda.synchronize()
    assert torch.equal(got, want)
    # one key more than the static scratch can hold is rejected, nothing runs
    assert fn(0, ctypes.c_void_p(got.data_ptr()), n + 1, ctypes.c_void_p(stream)) == mgs.MGS_ERR_INVALID
    assert b"static scratch" in lib.mgs_last_error_string()
    assert fn(3, ctypes.c_void_p(got.data_ptr()), MAX_KEYS[8] + 1, None) == mgs.MGS_ERR_INVALID


def test_noalloc_calls_allocate_no_device_memory(ctx, mgs):
    """The defining property: once the library's module is loaded on the GPU (the first call), further calls
    of every size and key width leave the device's free memory unchanged."""
    lib, fn = noalloc_fn(mgs)
    cases = [("u32", "uniform", 1 << 22), ("f32", "full-uniform-specials", 100_003), ("u64", "uniform", 1 << 21),
             ("i64", "zipf", 4097), ("u32", "uniform", 31)]
    bufs = [(mgs.dtype_code(dt), on_device(mgs.generate(dt, dist, 9, n)), n) for dt, dist, n in cases]
    stream = torch.cuda.current_stream().cuda_stream
    code, t, n = bufs[0]
    assert fn(code, ctypes.c_void_p(t.data_ptr()), n, ctypes.c_void_p(stream)) == mgs.MGS_OK  # warm-up call
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        for code, t, n in bufs:
            assert fn(code, ctypes.c_void_p(t.data_ptr()), n, ctypes.c_void_p(stream)) == mgs.MGS_OK, \
                lib.mgs_last_error_string()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free_before
