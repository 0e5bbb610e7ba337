"""GPU parity of the merge path: pivot search (FindPivot), two-way merge
(thrust::merge), k-way merge (HET sort's multiway merge) and TanasicSort over
g chunks of one GPU, against the oracle restatement of the reference."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]


def to_device(a):
    st = np.int32 if a.dtype.itemsize == 4 else np.int64
    return torch.from_numpy(np.ascontiguousarray(a).view(st).copy()).cuda()


def from_device(t, dt):
    return t.cpu().numpy().view(dt)


def keys(mgs, dtype, n, seed, dist="full-uniform"):
    dt = mgs.np_dtype(dtype)
    if dt.kind == "f" and dist in ("full-uniform", "zipf"):
        dist += "-specials"
    return mgs.generate(dt, dist, seed, n)


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("g", [2, 4, 8, 16])
@pytest.mark.parametrize("psize", [1, 7, 1000, 65536])
def test_find_pivot_matches_oracle(ctx, mgs, orc, dtype, g, psize):
    half = g // 2
    a = keys(mgs, dtype, g * psize, psize + g, "zipf" if psize > 7 else "full-uniform")
    left = orc.sort(a[: half * psize])
    right = orc.sort(a[half * psize:])
    parts = np.concatenate([left, right])
    want = orc.find_pivot(parts, psize, g)
    tl, tr = to_device(left), to_device(right)
    w = a.dtype.itemsize
    lp = [tl.data_ptr() + i * psize * w for i in range(half)]
    rp = [tr.data_ptr() + i * psize * w for i in range(half)]
    torch.cuda.synchronize()
    assert ctx.find_pivot_device(lp, rp, psize, dtype) == want


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("na,nb", [(0, 5), (5, 0), (1, 1), (4096, 4096), (4095, 4097), (100003, 7), (1 << 20, 777777)])
def test_merge_device_matches_oracle(ctx, mgs, orc, dtype, na, nb):
    a = orc.sort(keys(mgs, dtype, na, 1, "zipf"))
    b = orc.sort(keys(mgs, dtype, nb, 2, "zipf"))
    want = orc.merge(a, b)
    ta, tb = to_device(a), to_device(b)
    out = torch.empty(na + nb, dtype=ta.dtype, device="cuda")
    torch.cuda.synchronize()
    ctx.merge_device(ta.data_ptr(), na, tb.data_ptr(), nb, out.data_ptr(), dtype)
    ctx.synchronize()
    assert from_device(out, a.dtype).tobytes() == want.tobytes()


def test_merge_signed_zero_ties_first_range(ctx, mgs, orc):
    a = np.array([-0.0, -0.0, 1.0], np.float32)
    b = np.array([0.0, 0.0, 0.5], np.float32)
    ta, tb = to_device(a), to_device(b)
    out = torch.empty(6, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.merge_device(ta.data_ptr(), 3, tb.data_ptr(), 3, out.data_ptr(), "f32")
    ctx.synchronize()
    got = from_device(out, np.float32)
    assert list(np.signbit(got[:4])) == [True, True, False, False]
    assert got.tobytes() == orc.merge(a, b).tobytes()


def dirichlet_runs(mgs, orc, dtype, k, total, seed, dist="full-uniform"):
    rng = np.random.default_rng(seed)
    lens = rng.multinomial(total, rng.dirichlet(np.ones(k))) if k > 1 else np.array([total])
    return [orc.sort(keys(mgs, dtype, int(L), seed * 1000 + i, dist)) for i, L in enumerate(lens)]


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("k", [1, 2, 3, 8, 32, 64, 100])
@pytest.mark.parametrize("total", [1, 5000, 300001])
def test_kway_merge_matches_oracle(ctx, mgs, orc, dtype, k, total):
    runs = dirichlet_runs(mgs, orc, dtype, k, total, k + total % 97)
    want = orc.kway_merge(runs)
    dev = [to_device(r) for r in runs]
    out = torch.empty(total, dtype=dev[0].dtype, device="cuda")
    torch.cuda.synchronize()
    ctx.kway_merge_device([d.data_ptr() if d.numel() else 0 for d in dev], [r.size for r in runs], out.data_ptr(),
                          dtype)
    ctx.synchronize()
    assert from_device(out, runs[0].dtype).tobytes() == want.tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f32", "u64"])
@pytest.mark.parametrize("pattern", ["empty-between", "tiny-many", "equal-keys", "equal-keys-many"])
def test_kway_merge_empty_and_tiny_runs(ctx, mgs, orc, dtype, pattern):
    """Empty slices between non-empty ones, many runs of one to three keys, and equal keys in every run
    (ties must come out in run order): the per-tile pair walk of the merge rounds has to skip empty pairs.
    "equal-keys-many" has enough runs for 4-byte keys to take the sorted-tile path (and a tile range of
    zero: no pass at all)."""
    rng = np.random.default_rng(17)
    if pattern == "empty-between":
        lens = [0, 5, 0, 0, 3000, 0, 1, 0, 9000, 0, 0, 2, 0]
    elif pattern == "tiny-many":
        lens = list(rng.integers(0, 4, 1000))
    elif pattern == "equal-keys":
        lens = [4000, 0, 4001, 3, 4002, 0]
    else:
        lens = [int(x) for x in rng.integers(0, 3000, 40)]
    dist = "all-equal" if pattern.startswith("equal-keys") else "full-uniform"
    runs = [orc.sort(keys(mgs, dtype, int(L), 31 + i, dist)) for i, L in enumerate(lens)]
    if pattern.startswith("equal-keys") and dtype == "f32":  # equal keys with different bytes: -0.0 / +0.0 by run
        runs = [np.full(int(L), -0.0 if i % 2 == 0 else 0.0, dtype=np.float32) for i, L in enumerate(lens)]
    total = int(sum(lens))
    want = orc.kway_merge(runs)
    dev = [to_device(r) for r in runs]
    out = torch.empty(total, dtype=dev[0].dtype, device="cuda")
    torch.cuda.synchronize()
    ctx.kway_merge_device([d.data_ptr() if d.numel() else 0 for d in dev], [r.size for r in runs], out.data_ptr(),
                          dtype)
    ctx.synchronize()
    assert from_device(out, runs[0].dtype).tobytes() == want.tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f32", "u64"])
@pytest.mark.parametrize("k,dist", [(8, "full-uniform"), (64, "full-uniform"), (32, "zipf"), (5, "all-equal")])
def test_kway_merge_large_two_level_partition(ctx, mgs, orc, dtype, k, dist):
    total = 12_000_017  # > 512 tiles: the coarse partition level is used
    runs = dirichlet_runs(mgs, orc, dtype, k, total, 7, dist)
    want = orc.kway_merge(runs)
    dev = [to_device(r) for r in runs]
    out = torch.empty(total, dtype=dev[0].dtype, device="cuda")
    torch.cuda.synchronize()
    ctx.kway_merge_device([d.data_ptr() if d.numel() else 0 for d in dev], [r.size for r in runs], out.data_ptr(),
                          dtype)
    ctx.synchronize()
    assert from_device(out, runs[0].dtype).tobytes() == want.tobytes()


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("g", [2, 4, 8, 16])
@pytest.mark.parametrize("n", [1, 3, 8, 1000, 4099, 262147])
def test_tanasic_chunks_match_oracle(ctx, mgs, orc, dtype, g, n):
    a = keys(mgs, dtype, n, n + g, "zipf" if n > 100 else "full-uniform")
    want = orc.tanasic_sort(a, g)
    h = mgs.host_empty(n, a.dtype)
    h[:] = a
    ctx.tanasic_sort(h, g)
    assert h.tobytes() == want.tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f64"])
@pytest.mark.parametrize("g", [2, 8])
def test_tanasic_chunks_device_matches_oracle(ctx, mgs, orc, dtype, g):
    n = 1_000_003
    a = keys(mgs, dtype, n, 5)
    t = to_device(a)
    torch.cuda.synchronize()
    ctx.tanasic_sort_device(t.data_ptr(), n, dtype, g)
    assert from_device(t, a.dtype).tobytes() == orc.tanasic_sort(a, g).tobytes()


def test_tanasic_filler_defect_matches_reference_semantics(ctx, mgs, orc):
    a = np.array([np.inf, 1.0, 2.0, 3.0, 4.0], dtype=np.float32)
    h = mgs.host_empty(5, np.float32)
    h[:] = a
    ctx.tanasic_sort(h, 2)
    assert h.tobytes() == orc.tanasic_sort(a, 2).tobytes()
    assert h[-1] == np.finfo(np.float32).max


def test_tanasic_chunks_large_properties(ctx, mgs):
    n = 1 << 27
    g = torch.Generator(device="cuda")
    g.manual_seed(9)
    t = torch.randint(-2 ** 31, 2 ** 31 - 1, (n,), dtype=torch.int32, device="cuda", generator=g)
    s0 = t.to(torch.int64).sum().item()
    torch.cuda.synchronize()
    ctx.tanasic_sort_device(t.data_ptr(), n, "u32", 8)
    u = t.to(torch.int64) & 0xFFFFFFFF
    assert bool((u[1:] >= u[:-1]).all())
    assert t.to(torch.int64).sum().item() == s0
