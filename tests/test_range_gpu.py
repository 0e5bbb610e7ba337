"""GPU parity of the bit-range and descending sorts (mgs_sort_range_device),
keys only and with 4- or 8-byte values: bit-exact against the oracle and
against cub::DeviceRadixSort (SortKeys/SortPairs[Descending] with begin_bit /
end_bit) run on the same GPU from oracle/_ref."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]
VALUE_TYPES = {4: np.uint32, 8: np.uint64}


def to_device(a):
    st = np.int32 if a.dtype.itemsize == 4 else np.int64
    return torch.from_numpy(np.ascontiguousarray(a).view(st).copy()).cuda()


def from_device(t, dt):
    return t.cpu().numpy().view(dt)


def keys(mgs, dtype, n, seed):
    dt = mgs.np_dtype(dtype)
    return mgs.generate(dt, "full-uniform-specials" if dt.kind == "f" else "zipf", seed, n)


def ranges(bits):
    return [(0, bits), (0, 12), (4, bits - 3), (bits - 8, bits), (7, 7), (bits // 2, bits // 2 + 1)]


def engine(ctx, k, dtype, b, e, desc, v=None):
    tk = to_device(k)
    tv = to_device(v) if v is not None else None
    torch.cuda.synchronize()
    ctx.sort_range_device(tk.data_ptr(), k.size, dtype, b, e, desc, tv.data_ptr() if tv is not None else 0,
                          0 if v is None else v.dtype.itemsize)
    ctx.synchronize()
    gk = from_device(tk, k.dtype)
    return gk if v is None else (gk, from_device(tv, v.dtype))


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("vb", [0, 4, 8])
def test_range_sort_matches_oracle(ctx, mgs, orc, dtype, desc, vb):
    n = 70_001
    bits = mgs.np_dtype(dtype).itemsize * 8
    for i, (b, e) in enumerate(ranges(bits)):
        k = keys(mgs, dtype, n, 100 + i)
        if vb == 0:
            assert engine(ctx, k, dtype, b, e, desc).tobytes() == orc.sort_range(k, b, e, desc).tobytes()
        else:
            v = np.arange(n, dtype=VALUE_TYPES[vb])
            gk, gv = engine(ctx, k, dtype, b, e, desc, v)
            wk, wv = orc.sort_range(k, b, e, desc, v)
            assert gk.tobytes() == wk.tobytes() and gv.tobytes() == wv.tobytes(), (b, e)


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("desc", [False, True])
@pytest.mark.parametrize("vb", [0, 8])
def test_range_sort_matches_cub_on_gpu(ctx, mgs, orc, dtype, desc, vb):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    n = 200_003
    bits = mgs.np_dtype(dtype).itemsize * 8
    for i, (b, e) in enumerate([(0, bits), (3, bits - 5)]):
        k = keys(mgs, dtype, n, 7 + i)
        v = np.arange(n, dtype=np.uint64) if vb else None
        rk = to_device(k)
        rv = to_device(v) if vb else None
        torch.cuda.synchronize()
        orc.ref_cub_sort_range(orc.DTYPE_CODES[k.dtype], rk.data_ptr(), n, b, e, desc,
                               rv.data_ptr() if vb else 0, vb)
        got = engine(ctx, k, dtype, b, e, desc, v)
        if vb:
            assert got[0].tobytes() == from_device(rk, k.dtype).tobytes()
            assert got[1].tobytes() == from_device(rv, np.uint64).tobytes()
        else:
            assert got.tobytes() == from_device(rk, k.dtype).tobytes()


def test_full_range_ascending_equals_plain_sort(ctx, mgs, orc):
    k = keys(mgs, "f32", (1 << 20) + 9, 5)
    assert engine(ctx, k, "f32", 0, 32, False).tobytes() == orc.sort(k).tobytes()


def test_range_argument_errors(ctx, mgs):
    t = torch.zeros(8, dtype=torch.int32, device="cuda")
    for b, e in [(-1, 8), (9, 8), (0, 33)]:
        with pytest.raises(mgs.MgsError):
            ctx.sort_range_device(t.data_ptr(), 8, "u32", b, e)
    with pytest.raises(mgs.MgsError):
        ctx.sort_range_device(t.data_ptr(), 8, "u32", 0, 32, d_values=t.data_ptr(), value_bytes=2)
