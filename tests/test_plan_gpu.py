"""GPU parity of recorded sorts (mgs_plan_*): a device sort or a segmented sort
of fixed buffers recorded once into a CUDA graph and replayed on new contents of
the same buffers. Every replay is compared byte for byte with the oracle, and
the launch count of a replay with that of the direct call."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]


def storage(dt):
    return (np.int32, torch.int32) if dt.itemsize == 4 else (np.int64, torch.int64)


def keys(mgs, dtype, n, seed):
    dt = mgs.np_dtype(dtype)
    return mgs.generate(dt, "full-uniform-specials" if dt.kind == "f" else "zipf", seed, n)


def fill(t, a):
    t.copy_(torch.from_numpy(np.ascontiguousarray(a).view(storage(a.dtype)[0])))
    torch.cuda.synchronize()


def read(t, dt):
    return t.cpu().numpy().view(dt)


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("n", [1, 4097, 65537, (1 << 20) + 3])
def test_plan_sort_replays_match_oracle(ctx, mgs, orc, dtype, n):
    dt = mgs.np_dtype(dtype)
    t = torch.empty(n, dtype=storage(dt)[1], device="cuda")
    plan = ctx.plan_sort(t.data_ptr(), n, dtype)
    try:
        for seed in (1, 2):  # two replays on different contents of the same buffer
            a = keys(mgs, dtype, n, seed)
            fill(t, a)
            plan.launch()
            ctx.synchronize()
            assert read(t, dt).tobytes() == orc.sort(a).tobytes()
    finally:
        plan.close()


def test_plan_sort_with_caller_scratch_on_a_user_stream(ctx, mgs, orc):
    n = (1 << 18) + 77
    temp_bytes = mgs.Context.sort_temp_bytes("u64", n)
    temp = torch.empty(temp_bytes, dtype=torch.uint8, device="cuda")
    t = torch.empty(n, dtype=torch.int64, device="cuda")
    plan = ctx.plan_sort(t.data_ptr(), n, "u64", temp.data_ptr(), temp_bytes)
    s = torch.cuda.Stream()
    try:
        for seed in (3, 4):
            a = keys(mgs, "u64", n, seed)
            fill(t, a)
            plan.launch(s.cuda_stream)
            s.synchronize()
            ctx.synchronize()
            assert read(t, np.uint64).tobytes() == orc.sort(a).tobytes()
    finally:
        plan.close()
    with pytest.raises(mgs.MgsError):
        ctx.plan_sort(t.data_ptr(), n, "u64", temp.data_ptr(), temp_bytes // 2)


def test_plan_replay_launches_as_many_kernels_as_the_direct_call(ctx, mgs):
    n = 1 << 20
    t = torch.randint(-2 ** 31, 2 ** 31 - 1, (n,), dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    ctx.launch_count(reset=True)
    ctx.sort_device(t.data_ptr(), n, "u32")
    ctx.synchronize()
    direct = ctx.launch_count(reset=True)
    plan = ctx.plan_sort(t.data_ptr(), n, "u32")
    try:
        assert plan.launch_count() == direct
        plan.launch()
        ctx.synchronize()
        assert ctx.launch_count(reset=True) == direct
    finally:
        plan.close()


@pytest.mark.parametrize("dtype", ["u32", "f32", "u64", "f64"])
def test_plan_segmented_replays_match_oracle(ctx, mgs, orc, dtype):
    rng = np.random.default_rng(11)
    dt = mgs.np_dtype(dtype)
    tile = 16384 if dt.itemsize == 4 else 8192
    lengths = np.concatenate([[0, 1, 2, 255, 256, 257, tile - 1, tile + 1, 3 * tile],
                              rng.integers(0, 300, 300), rng.integers(300, tile, 20)])
    rng.shuffle(lengths)
    offs = np.zeros(len(lengths) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lengths)
    n = int(offs[-1])
    t = torch.empty(n, dtype=storage(dt)[1], device="cuda")
    o = torch.from_numpy(offs.view(np.int64)).cuda()
    plan = ctx.plan_segmented(t.data_ptr(), n, o.data_ptr(), len(lengths), dtype)
    try:
        for seed in (5, 6):
            a = keys(mgs, dtype, n, seed)
            fill(t, a)
            plan.launch()
            ctx.synchronize()
            assert read(t, dt).tobytes() == orc.segmented_sort(a, offs).tobytes()
    finally:
        plan.close()


def test_empty_plans_launch_nothing(ctx, mgs):
    t = torch.empty(1, dtype=torch.int32, device="cuda")
    for plan in (ctx.plan_sort(t.data_ptr(), 0, "u32"), ctx.plan_segmented(t.data_ptr(), 0, 0, 0, "u32")):
        assert plan.launch_count() == 0
        plan.launch()
        ctx.synchronize()
        plan.close()
    import ctypes
    lib = mgs.load_library()
    h = ctypes.c_void_p()
    rc = lib.mgs_plan_sort_create(ctx.handle, 99, ctypes.c_void_p(t.data_ptr()), 4, None, 0, ctypes.byref(h))
    assert rc == mgs.MGS_ERR_INVALID and not h.value
