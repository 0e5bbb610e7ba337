"""The C ABI library loads, exports every symbol include/*.h declares, and
reports errors as status codes (no GPU needed)."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

from conftest import ROOT


def declared_symbols():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(mgs_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return names


def test_library_exports_every_declared_symbol(mgs):
    lib = mgs.load_library()
    names = declared_symbols()
    assert len(names) >= 15
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_version_and_dtype_sizes(mgs):
    lib = mgs.load_library()
    assert lib.mgs_version() >= 100
    assert [lib.mgs_dtype_size(i) for i in range(6)] == [4, 4, 4, 8, 8, 8]
    assert lib.mgs_dtype_size(6) == 0 and lib.mgs_dtype_size(-1) == 0


def test_invalid_arguments_return_status(mgs):
    lib = mgs.load_library()
    assert lib.mgs_sort_temp_bytes(9, 10, ctypes.byref(ctypes.c_size_t())) == mgs.MGS_ERR_INVALID
    assert b"dtype" in lib.mgs_last_error_string()
    assert lib.mgs_sort_temp_bytes(0, 1 << 32, ctypes.byref(ctypes.c_size_t())) == mgs.MGS_ERR_INVALID
    assert lib.mgs_sort_device(None, 0, None, 10, None, 0, None) == mgs.MGS_ERR_INVALID
    assert lib.mgs_sort_host(None, 0, None, 10) == mgs.MGS_ERR_INVALID
    assert lib.mgs_generate(0, b"no-such-distribution", 1, ctypes.c_void_p(8), 4) == mgs.MGS_ERR_INVALID
    assert b"no-such-distribution" in lib.mgs_last_error_string()
    assert lib.mgs_generate(0, b"uniform-specials", 1, ctypes.c_void_p(8), 4) == mgs.MGS_ERR_INVALID


def test_temp_bytes_grow_with_n(mgs):
    small = mgs.Context.sort_temp_bytes("u32", 1000)
    big = mgs.Context.sort_temp_bytes("u32", 1 << 20)
    assert big > small >= 1000 * 4
    assert mgs.Context.sort_temp_bytes("u64", 1 << 20) > big


def test_context_without_gpu_fails_cleanly(mgs):
    if mgs.device_count() > 0:
        pytest.skip("a GPU is present")
    with pytest.raises(mgs.MgsError) as e:
        mgs.Context(0)
    assert e.value.code == mgs.MGS_ERR_NO_DEVICE
