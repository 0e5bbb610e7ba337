"""Failure detection, tested without a GPU fault.

* A bounded device-side wait that runs out: with one tile of the plain device
  sort held back (its look-back status is never published), the look-back of
  the next tile polls a word that nothing sets until its bound runs out. The
  sort still finishes, mgs_ctx_synchronize reports MGS_ERR_TIMEOUT, and the
  same context sorts bit-exactly afterwards.
* A device allocation that fails: the context arena's growth is made to fail
  as an out-of-memory cudaMalloc would; the call reports MGS_ERR_OOM, leaves
  the keys untouched, and the next call succeeds.
The reference has no such paths: its CheckCudaError ignores errors in release
builds (src/cuda_error.cuh:5-10).
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def _on_device(a):
    return torch.from_numpy(a.view(np.int32 if a.dtype.itemsize == 4 else np.int64).copy()).cuda()


@pytest.mark.gpu
@pytest.mark.parametrize("dtype,hold", [("u32", 3), ("u64", 0), ("f32", 17)])
def test_lookback_wait_runs_out_reports_timeout_and_context_recovers(mgs, orc, dtype, hold):
    n = (1 << 22) + 5
    a = mgs.generate(dtype, "full-uniform" + ("-specials" if dtype == "f32" else ""), 3, n)
    ctx = mgs.Context(0)
    try:
        d = _on_device(a)
        torch.cuda.synchronize()
        mgs.inject_waits(0, lookback_spins=64, hold_tile=hold)
        try:
            ctx.sort_device(d.data_ptr(), n, dtype)
            with pytest.raises(mgs.MgsError) as err:
                ctx.synchronize()
            assert err.value.code == mgs.MGS_ERR_TIMEOUT
            assert "look-back" in str(err.value)
        finally:
            mgs.inject_waits(0)  # default bounds, no tile held
        ctx.synchronize()  # the status was taken: the context is clean
        d = _on_device(a)
        torch.cuda.synchronize()
        ctx.sort_device(d.data_ptr(), n, dtype)
        ctx.synchronize()
        assert d.cpu().numpy().view(a.dtype).tobytes() == orc.sort(a).tobytes()
    finally:
        ctx.close()


@pytest.mark.gpu
def test_arena_allocation_failure_reports_oom_and_next_call_succeeds(mgs, orc):
    n = (1 << 20) + 3
    a = mgs.generate("u32", "full-uniform", 4, n)
    ctx = mgs.Context(0)  # a fresh context: its arena must grow on the first sort
    try:
        d = _on_device(a)
        torch.cuda.synchronize()
        mgs.inject_allocation_failures(1)
        try:
            with pytest.raises(mgs.MgsError) as err:
                ctx.sort_device(d.data_ptr(), n, "u32")
            assert err.value.code == mgs.MGS_ERR_OOM
        finally:
            mgs.inject_allocation_failures(0)
        assert ctx.arena_bytes() == 0
        assert d.cpu().numpy().view(np.uint32).tobytes() == a.tobytes()  # nothing ran
        ctx.sort_device(d.data_ptr(), n, "u32")
        ctx.synchronize()
        assert d.cpu().numpy().view(np.uint32).tobytes() == orc.sort(a).tobytes()
    finally:
        ctx.close()


def test_allocation_failure_hook_rejects_negative_counts(mgs):
    with pytest.raises(mgs.MgsError) as err:
        mgs.inject_allocation_failures(-1)
    assert err.value.code == mgs.MGS_ERR_INVALID
    mgs.inject_allocation_failures(0)
