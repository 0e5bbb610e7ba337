"""GPU parity of the engine's radix sort (mgs_sort_device / mgs_sort_host)
against the oracle and against the reference's own TanasicSort run on the same
GPU (oracle/_ref). Bit-exact: integer keys and IEEE keys including -0.0 and
NaN payloads."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]
SIZES = [1, 2, 3, 31, 255, 4095, 4096, 4097, 6145, 65537, 1 << 20, (1 << 22) + 13]
DISTS = ["uniform", "full-uniform", "normal0", "zipf", "all-equal", "sorted-full", "reverse-sorted-full",
         "nearly-sorted-swaps", "staggered", "bucket-sorted"]

_STORAGE = {4: (np.int32, torch.int32), 8: (np.int64, torch.int64)}


def to_device(a):
    st_np, _ = _STORAGE[a.dtype.itemsize]
    return torch.from_numpy(a.view(st_np).copy()).cuda()


def from_device(t, dt):
    return t.cpu().numpy().view(dt)


def keys_for(mgs, dtype, dist, n, seed=11):
    dt = mgs.np_dtype(dtype)
    if dt.kind == "f" and dist in ("full-uniform", "zipf", "normal0"):
        dist = dist + "-specials"
    if dist in ("staggered", "bucket-sorted") and n < 10:
        dist = "uniform"
    return mgs.generate(dt, dist, seed, n)


def device_sort(ctx, mgs, a, dtype, offset=0):
    t = to_device(np.concatenate([np.zeros(offset, a.dtype), a]) if offset else a)
    ptr = t.data_ptr() + offset * a.dtype.itemsize
    torch.cuda.synchronize()
    ctx.sort_device(ptr, a.size, dtype)
    ctx.synchronize()
    return from_device(t, a.dtype)[offset:]


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("n", SIZES)
def test_sort_device_uniform_sizes(ctx, mgs, orc, dtype, n):
    a = keys_for(mgs, dtype, "full-uniform", n)
    assert device_sort(ctx, mgs, a, dtype).tobytes() == orc.sort(a).tobytes()


@pytest.mark.parametrize("dtype,n", [
    ("u32", 16384 * 300), ("u32", 16384 * 300 + 1),        # 2^22 <= n < 2^26: 16384-key tiles
    ("f32", 16384 * 300 + 1), ("i64", 10240 * 500),        # 8-byte keys there: 10240-key tiles
    ("u64", 10240 * 500 + 1),
    ("u32", 20480 * 3300), ("u32", 20480 * 3300 + 1),      # n >= 2^26: 20480-key tiles
])
def test_sort_device_last_tile_full_or_one_key(ctx, mgs, orc, dtype, n):
    """The array's last tile places its keys from the bucket ends instead of looking back: a last tile that
    is full and one that holds a single key, for the tile sizes of the larger size classes."""
    a = keys_for(mgs, dtype, "full-uniform", n, seed=23)
    assert device_sort(ctx, mgs, a, dtype).tobytes() == orc.sort(a).tobytes()


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("dist", DISTS)
@pytest.mark.parametrize("n", [5000, 300001])
def test_sort_device_distributions(ctx, mgs, orc, dtype, dist, n):
    a = keys_for(mgs, dtype, dist, n)
    assert device_sort(ctx, mgs, a, dtype).tobytes() == orc.sort(a).tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f32", "u64", "f64"])
@pytest.mark.parametrize("offset", [1, 2, 3])
@pytest.mark.parametrize("n", [1, 5, 4097, 20481, 100003, 3 * 20480 + 5, 4 * 20480])
def test_sort_device_unaligned_keys(ctx, mgs, orc, dtype, offset, n):
    # keys not 16-byte aligned: tiles arrive as the 16-byte-aligned windows that cover them, read from an
    # offset in shared memory; a window that would leave the array (first or last tile) takes plain loads
    a = keys_for(mgs, dtype, "full-uniform", n)
    assert device_sort(ctx, mgs, a, dtype, offset=offset).tobytes() == orc.sort(a).tobytes()


@pytest.mark.parametrize("dtype", TYPES)
def test_sort_host_matches_oracle(ctx, mgs, orc, dtype):
    a = keys_for(mgs, dtype, "full-uniform", 777777)
    h = mgs.host_empty(a.size, a.dtype)
    h[:] = a
    ctx.sort_host(h)
    assert h.tobytes() == orc.sort(a).tobytes()


def test_sort_host_empty_returns_early(ctx, mgs):
    h = np.zeros(0, np.uint32)
    ctx.sort_host(h)


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("dist", ["uniform", "full-uniform", "normal", "sorted", "zero", "zipf"])
def test_sort_matches_reference_tanasic_sort_on_gpu(ctx, mgs, orc, dtype, dist):
    """The reference's own TanasicSort<T> (thrust::sort on this GPU) is the authority."""
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    a = keys_for(mgs, dtype, dist, 200003, seed=2147483647)
    ref = a.copy()
    orc.ref_tanasic_sort(ref, 0)
    assert device_sort(ctx, mgs, a, dtype).tobytes() == ref.tobytes()
    assert orc.sort(a).tobytes() == ref.tobytes()


def test_sort_large_properties(ctx, mgs):
    """2^28 u32 keys: sorted and a permutation of the input (sum, xor and count checks)."""
    n = 1 << 28
    g = torch.Generator(device="cuda")
    g.manual_seed(3)
    t = torch.randint(-2 ** 31, 2 ** 31 - 1, (n,), dtype=torch.int32, device="cuda", generator=g)
    s0 = t.to(torch.int64).sum().item()
    x0 = torch.bitwise_xor.reduce(t) if hasattr(torch.bitwise_xor, "reduce") else None
    h0 = torch.histc(t.float(), bins=64).cpu()
    torch.cuda.synchronize()
    ctx.sort_device(t.data_ptr(), n, "u32")
    ctx.synchronize()
    u = t.to(torch.int64) & 0xFFFFFFFF
    assert bool((u[1:] >= u[:-1]).all())
    assert t.to(torch.int64).sum().item() == s0
    assert torch.equal(torch.histc(t.float(), bins=64).cpu(), h0)
    del x0
