"""Byte-for-byte parity at the benchmark workloads' full sizes, on the GPU.

* 2^27 uint32 keys, the reference DataGenerator's "uniform" (seed 2147483647),
  sorted by mgs_sort_host (TanasicSort with one GPU) and mgs_sort_device:
  equal to the reference's own CPU sort (the gnu_parallel branch of
  src/sort_benchmark.cu:103-108, compiled into oracle/_ref).
* 2^30 keys of uint32, int32, float32 (0.1 % -0.0 and 0.1 % NaN) and uint64 over
  seven distributions (full-range uniform, normal(0, 2^20), Zipf(1.1) over 2^20
  values, sorted, reverse sorted, 1 % random swaps, all equal): equal to
  cub::DeviceRadixSort::SortKeys (the library the reference's thrust::sort
  dispatches to, src/tanasic_sort.cuh:264) on the same keys, on the same GPU.
* 2^30 uint32 uniform keys through mgs_sort_host: equal to the reference's own
  TanasicSort<uint32_t> with one GPU (src/tanasic_sort.cuh:223-299).
* 10^5 segments with Zipf(1.2) lengths in [1, 2^22] (about 2^28 keys, random
  order), uint32 and float32 (with -0.0 and NaN), one segmented-sort call: equal
  to the oracle's per-segment stable sort.
"""
import importlib.util
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

SEED = 2147483647
DISTS = ["full-uniform", "normal0", "zipf", "sorted-full", "reverse-sorted-full", "nearly-sorted-swaps",
         "all-equal"]
CODES = {"u32": 0, "i32": 1, "f32": 2, "u64": 3}
STORAGE = {4: (np.int32, torch.int32), 8: (np.int64, torch.int64)}
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _bench():
    """bench.py, for the batched workload's segment lengths (the same offsets the benchmark sorts)."""
    spec = importlib.util.spec_from_file_location("bench_workloads", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _release():
    torch.cuda.synchronize()
    torch.cuda.empty_cache()


def test_2p27_u32_uniform_matches_reference_cpu_sort(ctx, mgs, orc):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    n = 1 << 27
    a = orc.ref_generate(np.uint32, "uniform", SEED, n)
    assert np.array_equal(mgs.generate("u32", "uniform", SEED, n), a)  # the same input bytes
    ref = a.copy()
    orc.ref_gnu_parallel_sort(ref, orc.ref_num_procs())
    h = mgs.host_empty(n, np.uint32)
    h[:] = a
    ctx.sort_host(h)
    assert np.array_equal(h, ref)
    d = torch.from_numpy(a.view(np.int32)).cuda()
    torch.cuda.synchronize()
    ctx.sort_device(d.data_ptr(), n, "u32")
    ctx.synchronize()
    assert np.array_equal(d.cpu().numpy().view(np.uint32), ref)
    del d
    _release()


@pytest.mark.parametrize("dist", DISTS)
@pytest.mark.parametrize("dtype", ["u32", "i32", "f32", "u64"])
def test_2p30_matches_cub_radix_sort(ctx, mgs, orc, dtype, dist):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    n = 1 << 30
    w = 8 if dtype == "u64" else 4
    st_np, st_t = STORAGE[w]
    name = dist + ("-specials" if dtype == "f32" else "")
    src = torch.empty(n, dtype=st_t, device="cuda")
    if dist == "normal0":  # draws through the host C library's log: generated on the host
        src.copy_(torch.from_numpy(mgs.generate(dtype, name, SEED, n).view(st_np)))
    else:  # the host generator's bytes, generated on the device
        ctx.generate_device(src.data_ptr(), n, dtype, name, SEED)
    ctx.synchronize()
    if dtype == "f32" and dist != "all-equal":
        bits = src.to(torch.int64) & 0xFFFFFFFF
        assert int((bits == 0x80000000).sum()) > 0  # the case holds -0.0 ...
        assert int(((bits & 0x7FFFFFFF) > 0x7F800000).sum()) > 0  # ... and NaN
        del bits
    ours = src.clone()
    torch.cuda.synchronize()
    ctx.sort_device(ours.data_ptr(), n, dtype)
    ctx.synchronize()
    orc.ref_cub_sort(CODES[dtype], src.data_ptr(), n, w)  # src now holds the reference order
    assert torch.equal(ours, src)
    del ours, src
    _release()


def test_2p30_u32_uniform_matches_reference_tanasic_sort(ctx, mgs, orc):
    if not orc.ref_available():
        pytest.skip("oracle/_ref not built")
    n = 1 << 30
    a = orc.ref_generate(np.uint32, "uniform", SEED, n)
    ref = a.copy()
    orc.ref_tanasic_sort(ref, 0)
    h = mgs.host_empty(n, np.uint32)
    h[:] = a
    del a
    ctx.sort_host(h)
    assert np.array_equal(h, ref)
    _release()


@pytest.mark.parametrize("dtype", ["u32", "f32"])
def test_zipf_batch_of_1e5_segments_matches_oracle(ctx, mgs, orc, dtype):
    offs = _bench().zipf_segment_offsets(np.random.default_rng(11))
    n = int(offs[-1])
    a = mgs.generate(dtype, "full-uniform" + ("-specials" if dtype == "f32" else ""), 5, n)
    d = torch.from_numpy(a.view(np.int32).copy()).cuda()
    d_offs = torch.from_numpy(offs).cuda()
    torch.cuda.synchronize()
    ctx.segmented_sort_device(d.data_ptr(), n, d_offs.data_ptr(), offs.size - 1, dtype)
    ctx.synchronize()
    got = d.cpu().numpy().view(a.dtype)
    want = orc.segmented_sort(a, offs)
    assert got.tobytes() == want.tobytes()
    del d, d_offs
    _release()
