"""GPU parity of every onesweep variant (7 tile shapes x 2 ranking modes) on
multi-tile inputs with a partial last tile, for 4- and 8-byte keys, and of the
autotuner: it times every variant of the size classes it covers, keeps exactly
one per class, and sorts stay bit-exact afterwards."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture
def saved_table(mgs, tmp_path):
    path = tmp_path / "before.tune"
    mgs.tune_save(str(path))
    yield
    mgs.tune_load(str(path))


def device_sort(ctx, a, dtype):
    st = np.int32 if a.dtype.itemsize == 4 else np.int64
    t = torch.from_numpy(a.view(st).copy()).cuda()
    torch.cuda.synchronize()
    ctx.sort_device(t.data_ptr(), a.size, dtype)
    ctx.synchronize()
    return t.cpu().numpy().view(a.dtype)


@pytest.mark.parametrize("dtype", ["u32", "f32", "u64", "i64"])
@pytest.mark.parametrize("shape", range(7))
@pytest.mark.parametrize("mode", [2, 3])
def test_every_variant_matches_oracle(ctx, mgs, orc, saved_table, dtype, shape, mode):
    n = 100_003  # size class 1; 6-25 tiles depending on the shape, the last one partial
    mgs.tune_set(dtype, 1, shape, mode)
    assert mgs.tune_get(dtype, n) == (shape, mode)
    dt = mgs.np_dtype(dtype)
    a = mgs.generate(dt, "full-uniform-specials" if dt.kind == "f" else "zipf", shape * 10 + mode, n)
    assert device_sort(ctx, a, dtype).tobytes() == orc.sort(a).tobytes()


@pytest.mark.parametrize("dtype", ["u32", "u64"])
def test_autotune_keeps_one_variant_per_class(ctx, mgs, orc, saved_table, dtype):
    samples = ctx.autotune(dtype, 3 << 16, reps=2)  # size classes 0 and 1
    assert {s["size_class"] for s in samples} == {0, 1}
    for c in (0, 1):
        mine = [s for s in samples if s["size_class"] == c]
        assert len(mine) == 14 and all(s["ms"] > 0 for s in mine)
        chosen = [s for s in mine if s["chosen"]]
        assert len(chosen) == 1
        assert chosen[0]["ms"] == min(s["ms"] for s in mine)
        assert mgs.tune_get(dtype, mine[0]["n"]) == (chosen[0]["shape"], chosen[0]["rank_mode"])
    a = mgs.generate(dtype, "full-uniform", 3, 3 << 16)
    assert device_sort(ctx, a, dtype).tobytes() == orc.sort(a).tobytes()
