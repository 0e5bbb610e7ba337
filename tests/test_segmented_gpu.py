"""GPU parity of the batched segmented sort against the oracle: every segment
sorted on its own, stably, bit-exact; all size classes (warp, CTA, onesweep)
in one call; Zipf-distributed segment lengths like the batched workload."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]


def to_device(a):
    st = np.int32 if a.dtype.itemsize == 4 else np.int64
    return torch.from_numpy(np.ascontiguousarray(a).view(st).copy()).cuda()


def run_segmented(ctx, mgs, a, offsets, dtype):
    t = to_device(a)
    o = torch.from_numpy(np.asarray(offsets, dtype=np.int64)).cuda()
    torch.cuda.synchronize()
    ctx.segmented_sort_device(t.data_ptr(), a.size, o.data_ptr(), len(offsets) - 1, dtype)
    ctx.synchronize()
    return t.cpu().numpy().view(a.dtype)


def layout(rng, lengths):
    offs = np.zeros(len(lengths) + 1, dtype=np.uint64)
    offs[1:] = np.cumsum(lengths)
    return offs


@pytest.mark.parametrize("dtype", TYPES)
@pytest.mark.parametrize("seed", [1, 2])
def test_mixed_size_classes(ctx, mgs, orc, dtype, seed):
    rng = np.random.default_rng(seed)
    w = mgs.np_dtype(dtype).itemsize
    tile = 16384 if w == 4 else 8192
    lengths = np.concatenate([
        [0, 1, 2, 3, 31, 32, 33, 255, 256, 257],                 # warp class edges
        [tile - 1, tile, tile + 1, 2 * tile, 2 * tile + 1],       # CTA / onesweep edges
        rng.integers(0, 300, 200), rng.integers(300, tile, 20), rng.integers(tile, 5 * tile, 4),
    ])
    rng.shuffle(lengths)
    offs = layout(rng, lengths)
    n = int(offs[-1])
    dist = "full-uniform-specials" if mgs.np_dtype(dtype).kind == "f" else "zipf"
    a = mgs.generate(dtype, dist, seed, n)
    got = run_segmented(ctx, mgs, a, offs, dtype)
    assert got.tobytes() == orc.segmented_sort(a, offs).tobytes()


@pytest.mark.parametrize("dtype", TYPES)
def test_medium_segments_spread_over_warps(ctx, mgs, orc, dtype):
    """One-CTA segments of every length class: keys per lane 1, 2, ... up to a whole tile, the last
    warp's share partial or empty."""
    rng = np.random.default_rng(8)
    lengths = np.array([257, 300, 511, 512, 513, 1000, 1023, 1024, 1025, 2047, 2049, 4096, 5000, 8191, 8192,
                        8193, 12345, 16383, 16384] * 3)
    rng.shuffle(lengths)
    offs = layout(rng, lengths)
    n = int(offs[-1])
    dist = "full-uniform-specials" if mgs.np_dtype(dtype).kind == "f" else "zipf"
    a = mgs.generate(dtype, dist, 21, n)
    got = run_segmented(ctx, mgs, a, offs, dtype)
    assert got.tobytes() == orc.segmented_sort(a, offs).tobytes()


@pytest.mark.parametrize("dtype", ["u32", "f32", "u64"])
def test_zipf_segment_lengths(ctx, mgs, orc, dtype):
    """10^4 segments, Zipf(1.2) lengths in [1, 2^22] scaled to ~2^24 keys, random order."""
    rng = np.random.default_rng(5)
    lengths = np.minimum(rng.zipf(1.2, 10_000), 1 << 22).astype(np.float64)
    lengths = np.maximum(1, np.floor(lengths * ((1 << 24) / lengths.sum()))).astype(np.int64)
    offs = layout(rng, lengths)
    n = int(offs[-1])
    dist = "full-uniform-specials" if mgs.np_dtype(dtype).kind == "f" else "full-uniform"
    a = mgs.generate(dtype, dist, 9, n)
    got = run_segmented(ctx, mgs, a, offs, dtype)
    assert got.tobytes() == orc.segmented_sort(a, offs).tobytes()


@pytest.mark.parametrize("dtype", ["u32", "i64"])
def test_classify_rounds_and_histogram_ranges(ctx, mgs, orc, dtype):
    """Over 3 x 8192 segments, so the classification takes several rounds, with large segments placed at the
    round edges; more large tiles than SMs, so the histogram's per-CTA tile ranges start inside segments and
    cross several of them; segment starts at every alignment."""
    rng = np.random.default_rng(13)
    w = mgs.np_dtype(dtype).itemsize
    tile = 16384 if w == 4 else 8192
    nseg = 3 * 8192 + 5
    lengths = rng.integers(0, 300, nseg)
    for i, s in enumerate([0, 8191, 8192, 8193, 16383, 16384, 24575, 24576, nseg - 1]):
        lengths[s] = [tile + 1, 3 * tile + 7, 2 * tile, 40 * tile + 3, tile + 5, 7 * tile, 2 * tile + 1,
                      100 * tile - 1, 5 * tile + 2][i]
    offs = layout(rng, lengths)
    n = int(offs[-1])
    a = mgs.generate(dtype, "full-uniform", 17, n)
    got = run_segmented(ctx, mgs, a, offs, dtype)
    assert got.tobytes() == orc.segmented_sort(a, offs).tobytes()


def test_single_segment_equals_device_sort(ctx, mgs, orc):
    a = mgs.generate("u32", "uniform", 3, 1_000_003)
    got = run_segmented(ctx, mgs, a, [0, a.size], "u32")
    assert got.tobytes() == orc.sort(a).tobytes()


def test_all_equal_and_sorted_segments(ctx, mgs, orc):
    a = np.concatenate([np.full(40000, 7, np.uint32), np.arange(300, dtype=np.uint32),
                        np.arange(5000, 0, -1, dtype=np.uint32)])
    offs = [0, 40000, 40300, a.size]
    got = run_segmented(ctx, mgs, a, offs, "u32")
    assert got.tobytes() == orc.segmented_sort(a, np.array(offs)).tobytes()


def test_bad_offsets_reported(ctx, mgs):
    a = mgs.generate("u32", "uniform", 3, 1000)
    t = to_device(a)
    o = torch.tensor([0, 500, 400, 1000], dtype=torch.int64, device="cuda")
    torch.cuda.synchronize()
    ctx.segmented_sort_device(t.data_ptr(), a.size, o.data_ptr(), 3, "u32")
    with pytest.raises(mgs.MgsError) as e:
        ctx.synchronize()
    assert e.value.code == mgs.MGS_ERR_INVALID
    ctx.synchronize()  # the status word is cleared once reported
