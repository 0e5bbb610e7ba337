"""GPU parity of the device input generator (mgs_generate_device): for every
distribution it produces, the device buffer holds the same bytes as the host
generator (mgs_generate, pinned to the reference DataGenerator by the golden
hashes of test_data_generator.py) for the same dtype, seed and size. The
distributions that draw through the host C library's log / cos are refused."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]
DEVICE_DISTS = ["zero", "uniform", "sorted", "reverse-sorted", "staggered", "bucket-sorted", "full-uniform", "zipf",
                "sorted-full", "reverse-sorted-full", "nearly-sorted-swaps", "all-equal"]


def device_generate(ctx, mgs, dtype, dist, seed, n):
    dt = mgs.np_dtype(dtype)
    t = torch.zeros(max(n, 1), dtype=torch.int32 if dt.itemsize == 4 else torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.generate_device(t.data_ptr(), n, dtype, dist, seed)
    return t[:n].cpu().numpy().view(dt)


def first_difference(a, b):
    av = a.view(np.uint8).reshape(a.size, -1)
    bv = b.view(np.uint8).reshape(b.size, -1)
    diff = np.nonzero((av != bv).any(axis=1))[0]
    return (int(diff[0]), a[diff[0]], b[diff[0]]) if diff.size else None


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("dist", DEVICE_DISTS)
@pytest.mark.parametrize("n", [1, 9, 10, 19, 4097, 100_003])
def test_device_generator_matches_host(ctx, mgs, dtype, dist, n):
    seed = 1000 + n
    host = mgs.generate(dtype, dist, seed, n)
    dev = device_generate(ctx, mgs, dtype, dist, seed, n)
    assert dev.tobytes() == host.tobytes(), first_difference(dev, host)


@pytest.mark.parametrize("dtype", ["f32", "f64"])
@pytest.mark.parametrize("dist", ["full-uniform", "zipf", "uniform", "sorted-full", "nearly-sorted-swaps",
                                  "all-equal"])
def test_device_generator_specials_match_host(ctx, mgs, dtype, dist):
    n = 300_007
    host = mgs.generate(dtype, dist + "-specials", 77, n)
    dev = device_generate(ctx, mgs, dtype, dist + "-specials", 77, n)
    assert dev.tobytes() == host.tobytes(), first_difference(dev, host)


@pytest.mark.parametrize("dtype,dist", [("u32", "uniform"), ("f32", "staggered"), ("u64", "full-uniform"),
                                        ("i32", "zipf"), ("f64", "bucket-sorted"), ("u32", "nearly-sorted-swaps"),
                                        ("i64", "reverse-sorted")])
def test_device_generator_large_matches_host(ctx, mgs, dtype, dist):
    """2^24 + 3 keys: 128 mt19937 streams of 131072 values, a 167772-swap replay, sorted buckets."""
    n = (1 << 24) + 3
    host = mgs.generate(dtype, dist, 2024, n)
    dev = device_generate(ctx, mgs, dtype, dist, 2024, n)
    assert dev.tobytes() == host.tobytes(), first_difference(dev, host)


def test_device_generator_seeds_differ(ctx, mgs):
    a = device_generate(ctx, mgs, "u32", "uniform", 1, 4096)
    b = device_generate(ctx, mgs, "u32", "uniform", 2, 4096)
    assert a.tobytes() != b.tobytes()


def test_device_generator_refusals(ctx, mgs):
    t = torch.zeros(64, dtype=torch.int64, device="cuda")
    for dist in ["normal", "nearly-sorted", "normal0", "no-such-distribution"]:
        with pytest.raises(mgs.MgsError):
            ctx.generate_device(t.data_ptr(), 64, "u64", dist, 1)
    with pytest.raises(mgs.MgsError):
        ctx.generate_device(t.data_ptr(), 64, "u64", "uniform-specials", 1)  # -specials is for f32 / f64
    with pytest.raises(mgs.MgsError):
        ctx.generate_device(t.data_ptr() + 4, 8, "u64", "uniform", 1)  # not 8-byte aligned
    ctx.generate_device(t.data_ptr(), 0, "u64", "uniform", 1)  # nothing to do
    assert int(t.abs().sum()) == 0
