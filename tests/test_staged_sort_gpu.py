"""GPU parity of the staged host sort: mgs_sort_host from 2^24 keys up copies
the keys in slabs, sorts each slab as it lands, merges the sorted slabs window
by window and copies each window back while the next is merged. Bit-exact
against the oracle (IEEE keys with -0.0 and NaN payloads check that equal keys
keep their input order across the slab merge)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]


def keys_for(mgs, dtype, dist, n, seed=5):
    dt = mgs.np_dtype(dtype)
    if dt.kind == "f" and dist in ("full-uniform", "zipf", "normal0"):
        dist = dist + "-specials"
    return mgs.generate(dt, dist, seed, n)


def pinned_copy(mgs, a):
    h = mgs.host_empty(a.size, a.dtype)
    h[:] = a
    return h


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("n", [1 << 24, (1 << 24) + 4097])
def test_staged_sort_host_matches_oracle(ctx, mgs, orc, dtype, n):
    a = keys_for(mgs, dtype, "full-uniform", n)
    h = pinned_copy(mgs, a)
    ctx.sort_host(h)
    assert h.tobytes() == orc.sort(a).tobytes()


@pytest.mark.parametrize("dist", ["zipf", "all-equal", "sorted-full", "reverse-sorted-full", "nearly-sorted-swaps",
                                  "normal0"])
@pytest.mark.parametrize("dtype", ["u32", "f32", "f64"])
def test_staged_sort_host_distributions(ctx, mgs, orc, dtype, dist):
    a = keys_for(mgs, dtype, dist, (1 << 25) + 3)
    h = pinned_copy(mgs, a)
    ctx.sort_host(h)
    assert h.tobytes() == orc.sort(a).tobytes()


def test_staged_sort_host_pageable_buffer(ctx, mgs, orc):
    """A pageable (not pinned) buffer takes the same path; the copies then do not overlap."""
    a = keys_for(mgs, "u64", "full-uniform", (1 << 24) + 77)
    h = a.copy()
    ctx.sort_host(h)
    assert h.tobytes() == orc.sort(a).tobytes()


def test_staged_sort_host_twice_in_a_row(ctx, mgs, orc):
    """A second call reuses the grown arena and its scratch state."""
    for seed in (1, 2):
        a = keys_for(mgs, "i32", "full-uniform", (1 << 24) + 999, seed=seed)
        h = pinned_copy(mgs, a)
        ctx.sort_host(h)
        assert h.tobytes() == orc.sort(a).tobytes()


def test_staged_sort_host_large_properties(ctx, mgs):
    """2^28 u32 keys through the host path: ascending and a permutation of the input."""
    n = 1 << 28
    rng = np.random.default_rng(9)
    h = mgs.host_empty(n, np.uint32)
    h[:] = rng.integers(0, 1 << 32, n, dtype=np.uint32)
    s0 = int(h.sum(dtype=np.uint64))
    x0 = int(np.bitwise_xor.reduce(h))
    c0 = np.bincount(h >> 24, minlength=256)
    ctx.sort_host(h)
    assert bool((h[1:] >= h[:-1]).all())
    assert int(h.sum(dtype=np.uint64)) == s0
    assert int(np.bitwise_xor.reduce(h)) == x0
    assert np.array_equal(np.bincount(h >> 24, minlength=256), c0)
