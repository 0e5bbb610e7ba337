"""The serving loop: mixed request sizes and key types from several threads,
continuous batching with coalescing; every result equals the oracle and is the
same alone and in the mix; cancellation, admission limits and statistics."""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TYPES = ["u32", "i32", "f32", "u64"]


def make_requests(mgs, seed, count, max_log2=17):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        dtype = TYPES[rng.integers(0, len(TYPES))]
        n = int(2 ** rng.uniform(0, max_log2))
        dist = "full-uniform-specials" if dtype == "f32" else "full-uniform"
        a = mgs.generate(dtype, dist, seed * 1000 + i, n)
        h = mgs.host_empty(n, a.dtype)
        h[:] = a
        out.append((a, h))
    return out


def test_mixed_requests_match_oracle_and_alone(mgs, orc):
    reqs = make_requests(mgs, 1, 300)
    srv = mgs.Server(0, num_slots=4, slot_keys=1 << 22, coalesce_keys=1 << 14)
    try:
        ids = [srv.submit(h) for _, h in reqs]
        assert all(srv.wait(i) == mgs.MGS_OK for i in ids)
        for a, h in reqs:
            assert h.tobytes() == orc.sort(a).tobytes()
        st = srv.stats()
        assert st["completed"] == len(reqs) and st["batches"] < len(reqs)  # small requests were coalesced
        assert st["p99_us"] >= st["p50_us"] > 0
        # the same requests one at a time give the same bytes
        for a, h_mix in reqs[:40]:
            h = mgs.host_empty(a.size, a.dtype)
            h[:] = a
            assert srv.wait(srv.submit(h)) == mgs.MGS_OK
            assert h.tobytes() == h_mix.tobytes()
    finally:
        srv.close()


def test_concurrent_submitters(mgs, orc):
    srv = mgs.Server(0, num_slots=3, slot_keys=1 << 21, coalesce_keys=1 << 12)
    errors = []

    def worker(seed):
        try:
            reqs = make_requests(mgs, seed, 60, max_log2=15)
            ids = [srv.submit(h) for _, h in reqs]
            for i in ids:
                assert srv.wait(i) == mgs.MGS_OK
            for a, h in reqs:
                assert h.tobytes() == orc.sort(a).tobytes()
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    threads = [threading.Thread(target=worker, args=(s,)) for s in range(10, 14)]
    [t.start() for t in threads]
    [t.join() for t in threads]
    srv.close()
    assert not errors, errors


def test_plain_form_one_request_per_launch(mgs, orc):
    reqs = make_requests(mgs, 3, 40, max_log2=14)
    srv = mgs.Server(0, num_slots=1, slot_keys=1 << 20, coalesce_keys=0)
    try:
        ids = [srv.submit(h) for _, h in reqs]
        assert all(srv.wait(i) == mgs.MGS_OK for i in ids)
        for a, h in reqs:
            assert h.tobytes() == orc.sort(a).tobytes()
        st = srv.stats()
        assert st["batches"] == sum(1 for a, _ in reqs if a.size > 1)
    finally:
        srv.close()


def test_limits_cancel_and_timeout(mgs):
    srv = mgs.Server(0, num_slots=1, slot_keys=1 << 16, coalesce_keys=0)
    try:
        big = mgs.host_empty((1 << 16) + 1, np.uint64)
        with pytest.raises(mgs.MgsError) as e:
            srv.submit(big)
        assert e.value.code == mgs.MGS_ERR_INVALID
        # keep the single slot busy, then cancel a queued request
        keys = [mgs.host_empty(1 << 16, np.uint32) for _ in range(20)]
        for k in keys:
            k[:] = np.arange(k.size, 0, -1, dtype=np.uint32)
        ids = [srv.submit(k) for k in keys]
        cancelled = 0
        for i in reversed(ids):
            try:
                srv.cancel(i)
                cancelled += 1
            except mgs.MgsError as err:
                assert err.code == mgs.MGS_ERR_BUSY
        statuses = [srv.wait(i) for i in ids]
        assert statuses.count(mgs.MGS_ERR_CANCELLED) == cancelled >= 1
        for k, s in zip(keys, statuses):
            if s == mgs.MGS_OK:
                assert np.all(k[1:] >= k[:-1])
        assert srv.stats()["cancelled"] == cancelled
    finally:
        srv.close()


torch = pytest.importorskip("torch")
DEVICE_TYPES = ["u32", "i32", "f32", "u64", "i64", "f64"]


def device_requests(mgs, seed, count, max_log2=17):
    """(input copy on the host, device tensor holding the same keys) per request: mixed types and sizes."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        dtype = DEVICE_TYPES[rng.integers(0, len(DEVICE_TYPES))]
        n = int(2 ** rng.uniform(0, max_log2))
        dist = "full-uniform-specials" if dtype in ("f32", "f64") else "full-uniform"
        a = mgs.generate(dtype, dist, seed * 1000 + i, n)
        st = np.int32 if a.dtype.itemsize == 4 else np.int64
        out.append((a, torch.from_numpy(a.view(st).copy()).cuda()))
    torch.cuda.synchronize()
    return out


def test_device_requests_match_oracle_alone_and_in_mix(mgs, orc):
    reqs = device_requests(mgs, 21, 240)
    srv = mgs.Server(0, num_slots=4, coalesce_keys=1 << 14)
    try:
        ids = [srv.submit_device(t.data_ptr(), a.size, a.dtype, keep=t) for a, t in reqs]
        assert all(srv.wait(i) == mgs.MGS_OK for i in ids)
        mixed = [t.cpu().numpy().view(a.dtype) for a, t in reqs]
        for (a, _), got in zip(reqs, mixed):
            assert got.tobytes() == orc.sort(a).tobytes()
        assert srv.stats()["batches"] < len(reqs)
        # alone, one at a time, each request gives the same bytes as in the mix
        for (a, _), got in list(zip(reqs, mixed))[:60]:
            st = np.int32 if a.dtype.itemsize == 4 else np.int64
            t = torch.from_numpy(a.view(st).copy()).cuda()
            torch.cuda.synchronize()
            assert srv.wait(srv.submit_device(t.data_ptr(), a.size, a.dtype, keep=t)) == mgs.MGS_OK
            assert t.cpu().numpy().view(a.dtype).tobytes() == got.tobytes()
    finally:
        srv.close()


def test_uint32_and_int32_requests_share_one_batch(mgs, orc):
    """Small uint32 and int32 requests are sorted by one segmented launch: the int32 keys with their top bit
    inverted on the way in and out, which must still give int32 order."""
    reqs = []
    for i in range(64):
        dtype = "i32" if i % 2 else "u32"
        a = mgs.generate(dtype, "full-uniform", 500 + i, 1000 + 37 * i)
        h = mgs.host_empty(a.size, a.dtype)
        h[:] = a
        reqs.append((a, h))
    srv = mgs.Server(0, num_slots=1, coalesce_keys=1 << 16)
    try:
        blocker = mgs.host_empty(1 << 24, np.uint32)  # keeps the only stream busy while the small ones queue
        blocker[:] = mgs.generate("u32", "full-uniform", 1, blocker.size)
        first = srv.submit(blocker)
        ids = [srv.submit(h) for _, h in reqs]
        assert srv.wait(first) == mgs.MGS_OK
        assert all(srv.wait(i) == mgs.MGS_OK for i in ids)
        for a, h in reqs:
            assert h.tobytes() == orc.sort(a).tobytes()
        assert srv.stats()["batches"] <= 3  # the blocker, then the queued small requests together
    finally:
        srv.close()


def test_mixed_host_and_device_requests_in_one_batch(mgs, orc):
    reqs_h = make_requests(mgs, 31, 30, max_log2=12)
    reqs_d = device_requests(mgs, 32, 30, max_log2=12)
    srv = mgs.Server(0, num_slots=1, coalesce_keys=1 << 12)
    try:
        ids = []
        for (ah, h), (ad, t) in zip(reqs_h, reqs_d):
            ids.append(srv.submit(h))
            ids.append(srv.submit_device(t.data_ptr(), ad.size, ad.dtype, keep=t))
        assert all(srv.wait(i) == mgs.MGS_OK for i in ids)
        for a, h in reqs_h:
            assert h.tobytes() == orc.sort(a).tobytes()
        for a, t in reqs_d:
            assert t.cpu().numpy().view(a.dtype).tobytes() == orc.sort(a).tobytes()
    finally:
        srv.close()


def test_admission_by_free_pool_memory(mgs, orc):
    """A small pool: requests queue until earlier batches give their bytes back; one that could never fit is
    refused at submission; the pool is whole again when everything is done."""
    pool = 96 << 20
    srv = mgs.Server(0, num_slots=4, coalesce_keys=0, device_budget_bytes=pool)
    try:
        n = 3 << 20  # ~12 MB of keys + ~13 MB of scratch as a host request: three fit at a time
        reqs = []
        for i in range(12):
            a = mgs.generate("u32", "full-uniform", 700 + i, n)
            h = mgs.host_empty(n, np.uint32)
            h[:] = a
            reqs.append((a, h))
        ids = [srv.submit(h) for _, h in reqs]
        assert all(srv.wait(i) == mgs.MGS_OK for i in ids)
        for a, h in reqs:
            assert h.tobytes() == orc.sort(a).tobytes()
        huge = mgs.host_empty(16 << 20, np.uint64)
        with pytest.raises(mgs.MgsError) as e:
            srv.submit(huge)
        assert e.value.code == mgs.MGS_ERR_INVALID
        st = srv.stats()
        assert st["pool_bytes"] == pool and st["pool_free_bytes"] == pool and st["rejected"] == 1
    finally:
        srv.close()
