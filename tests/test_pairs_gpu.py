"""GPU parity of the key-value sort and argsort (mgs_sort_pairs_device,
mgs_argsort_device): keys bit-exact as by the keys-only sort and values moved
with their keys, equal keys (including -0.0 / +0.0) in input order; checked
against the oracle and against thrust::sort_by_key from the library the
reference sorts with, run on the same GPU (oracle/_ref)."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]
VALUE_TYPES = {4: np.uint32, 8: np.uint64}


def keys(mgs, dtype, n, seed, dist=None):
    dt = mgs.np_dtype(dtype)
    if dist is None:
        dist = "full-uniform-specials" if dt.kind == "f" else "zipf"
    return mgs.generate(dt, dist, seed, n)


def to_device(a):
    st = np.int32 if a.dtype.itemsize == 4 else np.int64
    return torch.from_numpy(np.ascontiguousarray(a).view(st).copy()).cuda()


def from_device(t, dt):
    return t.cpu().numpy().view(dt)


def values(n, vb, seed):
    return np.random.default_rng(seed).integers(0, np.iinfo(VALUE_TYPES[vb]).max, n, dtype=VALUE_TYPES[vb],
                                                endpoint=True)


def engine_pairs(ctx, k, v, dtype):
    tk, tv = to_device(k), to_device(v)
    torch.cuda.synchronize()
    ctx.sort_pairs_device(tk.data_ptr(), tv.data_ptr(), v.dtype.itemsize, k.size, dtype)
    ctx.synchronize()
    return from_device(tk, k.dtype), from_device(tv, v.dtype)


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("vb", [4, 8])
@pytest.mark.parametrize("n", [1, 7, 4097, 65537, (1 << 20) + 3])
def test_sort_pairs_matches_oracle(ctx, mgs, orc, dtype, vb, n):
    k = keys(mgs, dtype, n, n % 1000 + vb)
    v = values(n, vb, n)
    gk, gv = engine_pairs(ctx, k, v, dtype)
    wk, wv = orc.sort_pairs(k, v)
    assert gk.tobytes() == wk.tobytes()
    assert gv.tobytes() == wv.tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f32", "u64", "f64"])
@pytest.mark.parametrize("dist", ["all-equal", "sorted-full", "reverse-sorted-full", "zipf"])
def test_sort_pairs_distributions(ctx, mgs, orc, dtype, dist):
    """All-equal keys skip every pass (values stay in place); sorted inputs; heavy duplicates."""
    n = 300_007
    dt = mgs.np_dtype(dtype)
    k = keys(mgs, dtype, n, 9, dist + ("-specials" if dt.kind == "f" and dist == "zipf" else ""))
    v = values(n, 4, 9)
    gk, gv = engine_pairs(ctx, k, v, dtype)
    wk, wv = orc.sort_pairs(k, v)
    assert gk.tobytes() == wk.tobytes() and gv.tobytes() == wv.tobytes()


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("vb", [4, 8])
def test_sort_pairs_matches_thrust_sort_by_key_on_gpu(ctx, mgs, orc, dtype, vb):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    n = 200_003
    k = keys(mgs, dtype, n, 21)
    v = values(n, vb, 21)
    rk, rv = to_device(k), to_device(v)
    torch.cuda.synchronize()
    orc.ref_thrust_sort_by_key(orc.DTYPE_CODES[k.dtype], rk.data_ptr(), rv.data_ptr(), vb, n)
    ref_k, ref_v = from_device(rk, k.dtype), from_device(rv, v.dtype)
    gk, gv = engine_pairs(ctx, k, v, dtype)
    assert gk.tobytes() == ref_k.tobytes() and gv.tobytes() == ref_v.tobytes()
    wk, wv = orc.sort_pairs(k, v)
    assert wk.tobytes() == ref_k.tobytes() and wv.tobytes() == ref_v.tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f32", "i64", "f64"])
@pytest.mark.parametrize("ib", [4, 8])
def test_argsort_matches_oracle(ctx, mgs, orc, dtype, ib):
    n = (1 << 18) + 5
    k = keys(mgs, dtype, n, 33)
    tk = to_device(k)
    ti = torch.empty(n, dtype=torch.int32 if ib == 4 else torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.argsort_device(tk.data_ptr(), ti.data_ptr(), ib, n, dtype)
    ctx.synchronize()
    idx = from_device(ti, VALUE_TYPES[ib])
    wk, wi = orc.sort_pairs(k, np.arange(n, dtype=VALUE_TYPES[ib]))
    assert from_device(tk, k.dtype).tobytes() == wk.tobytes()
    assert idx.tobytes() == wi.tobytes()
    assert k[idx.astype(np.int64)].tobytes() == wk.tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f64"])
@pytest.mark.parametrize("vb", [4, 8])
@pytest.mark.parametrize("koff,voff", [(1, 0), (0, 1), (3, 1), (2, 3)])
@pytest.mark.parametrize("n", [3, 8193, 3 * 16384 + 77])
def test_sort_pairs_unaligned_buffers(ctx, mgs, orc, dtype, vb, koff, voff, n):
    """Keys and values at element offsets that are not 16-byte aligned (each on its own shift)."""
    k = keys(mgs, dtype, n, 51)
    v = values(n, vb, 52)
    tk = to_device(np.concatenate([np.zeros(koff, k.dtype), k]))
    tv = to_device(np.concatenate([np.zeros(voff, v.dtype), v]))
    torch.cuda.synchronize()
    ctx.sort_pairs_device(tk.data_ptr() + koff * k.dtype.itemsize, tv.data_ptr() + voff * vb, vb, n, dtype)
    ctx.synchronize()
    wk, wv = orc.sort_pairs(k, v)
    assert from_device(tk, k.dtype)[koff:].tobytes() == wk.tobytes()
    assert from_device(tv, v.dtype)[voff:].tobytes() == wv.tobytes()


def test_sort_pairs_large_argsort_properties(ctx, mgs):
    """2^26 u32 keys: the argsort's indices gather the input into ascending order, ties by position."""
    n = 1 << 26
    g = torch.Generator(device="cuda")
    g.manual_seed(4)
    src = torch.randint(0, 1 << 20, (n,), dtype=torch.int32, device="cuda", generator=g)  # many equal keys
    t = src.clone()
    idx = torch.empty(n, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.argsort_device(t.data_ptr(), idx.data_ptr(), 4, n, "u32")
    ctx.synchronize()
    gathered = src[idx.to(torch.int64)]
    assert torch.equal(gathered, t)
    assert bool((t[1:] >= t[:-1]).all())
    same = t[1:] == t[:-1]
    assert bool((idx[1:][same] > idx[:-1][same]).all())  # stable: equal keys keep their input order


def test_sort_pairs_argument_errors(ctx, mgs):
    k = torch.zeros(16, dtype=torch.int32, device="cuda")
    v = torch.zeros(32, dtype=torch.int32, device="cuda")
    with pytest.raises(mgs.MgsError):
        ctx.sort_pairs_device(k.data_ptr(), v.data_ptr(), 2, 16, "u32")
    with pytest.raises(mgs.MgsError):
        ctx.sort_pairs_device(k.data_ptr(), v.data_ptr() + 4, 8, 8, "u32")  # values not 8-byte aligned
    with pytest.raises(mgs.MgsError):
        ctx.sort_pairs_device(k.data_ptr(), 0, 4, 16, "u32")
    ctx.sort_pairs_device(k.data_ptr(), v.data_ptr(), 4, 0, "u32")  # empty: nothing to do
    lib = mgs.load_library()
    b = ctypes.c_size_t()
    assert lib.mgs_sort_pairs_temp_bytes(0, 4, 1000, ctypes.byref(b)) == 0 and b.value > 0
