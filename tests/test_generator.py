"""The engine's DataGenerator reproduces the reference's (src/data_generator.cuh)
byte for byte, pinned by golden hashes taken from the reference itself and,
where oracle/_ref is built, by a direct comparison."""
import hashlib
import json
import os
import sys

import numpy as np
import pytest

from conftest import ROOT

sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
import make_golden  # noqa: E402

GOLDEN = json.load(open(os.path.join(ROOT, "tests", "golden", "generator.json")))["entries"]


@pytest.mark.parametrize("entry", GOLDEN, ids=lambda e: f"{e['dtype']}-{e['distribution']}-{e['n']}-{e['seed']}")
def test_generator_matches_reference_golden(mgs, entry):
    a = mgs.generate(np.dtype(entry["dtype"]), entry["distribution"], entry["seed"], entry["n"])
    assert make_golden.digest(a, entry["distribution"]) == entry["sha256"]


def test_nearly_sorted_differs_only_at_race_positions(mgs, orc):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    n = 100003
    a = mgs.generate(np.uint32, "nearly-sorted", 2147483647, n)
    b = orc.ref_generate(np.uint32, "nearly-sorted", 2147483647, n)
    diff = np.nonzero(a != b)[0]
    assert set(diff.tolist()) <= set(make_golden.race_positions(n).tolist())


@pytest.mark.parametrize("dtype", ["u32", "i32", "f32", "u64", "i64", "f64"])
def test_reference_default_case_matches_directly(mgs, orc, dtype):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    dt = mgs.np_dtype(dtype)
    for dist in ["uniform", "normal", "staggered", "bucket-sorted", "reverse-sorted"]:
        a = mgs.generate(dt, dist, 2147483647, 40000)
        b = orc.ref_generate(dt, dist, 2147483647, 40000)
        assert a.tobytes() == b.tobytes(), dist


def test_generator_blocks_do_not_depend_on_n(mgs):
    # Generator thread 0 owns a leading block of at least 1000 keys for both
    # sizes, so the first 1000 keys are the same draws of the same mt19937.
    a = mgs.generate(np.int32, "uniform", 2147483647, 10 ** 6)
    b = mgs.generate(np.int32, "uniform", 2147483647, 1 << 22)
    assert np.array_equal(a[:1000], b[:1000])
    assert a.min() >= 0  # the reference's int uniform is [0, INT_MAX) (src/data_generator.cuh:45)


@pytest.mark.parametrize("dtype", ["u32", "i32", "f32", "u64", "i64", "f64"])
def test_workload_distributions(mgs, orc, dtype):
    dt = mgs.np_dtype(dtype)
    n = 200000
    full = mgs.generate(dt, "full-uniform", 1, n)
    assert np.array_equal(full, mgs.generate(dt, "full-uniform", 1, n))  # deterministic
    if dt.kind in "iu":
        assert full.min() < np.iinfo(dt).min // 2 + np.iinfo(dt).max // 4
        assert full.max() > np.iinfo(dt).max // 2
    else:
        assert (full < 0).any() and (full > 0).any()
    z = mgs.generate(dt, "zipf", 1, n)
    assert len(np.unique(z)) < n // 4
    s = mgs.generate(dt, "sorted-full", 1, n)
    assert np.array_equal(orc.order_keys(s), np.sort(orc.order_keys(s)))
    r = mgs.generate(dt, "reverse-sorted-full", 1, n)
    assert np.array_equal(orc.order_keys(r), np.sort(orc.order_keys(r))[::-1])
    ns = mgs.generate(dt, "nearly-sorted-swaps", 1, n)
    assert 0 < np.count_nonzero(ns != s) <= 2 * (n // 100)
    e = mgs.generate(dt, "all-equal", 1, n)
    assert (e == e[0]).all()
    nm = mgs.generate(dt, "normal0", 1, n)
    if dt.kind == "f":
        assert abs(float(np.median(nm))) < 2 ** 16
        sp = mgs.generate(dt, "full-uniform-specials", 3, n)
        bits = sp.view(np.uint32 if dt.itemsize == 4 else np.uint64)
        neg0 = np.count_nonzero(bits == (np.uint64(1) << np.uint64(dt.itemsize * 8 - 1)).astype(bits.dtype))
        nans = np.count_nonzero(np.isnan(sp))
        assert 0.0005 * n < neg0 < 0.002 * n and 0.0005 * n < nans < 0.002 * n
        assert (np.signbit(sp[np.isnan(sp)])).any() and (~np.signbit(sp[np.isnan(sp)])).any()
