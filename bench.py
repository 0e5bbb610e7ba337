"""Benchmark of the plain single-GPU sort path (2^30 uint32 keys).

python bench.py [--gpus N --steps K --warmup W] [--impl mgs|reference]

One step = one in-place sort of 2^30 uint32 keys drawn by the reference's
DataGenerator ("uniform" over [0, 2^32), seed 2147483647). Per rank:
  value : keys/s of mgs_sort_device with the keys resident in HBM. Each step's
          input is restored from a pristine device copy before the step, outside
          its CUDA-event timed region; inputs (4 GiB) exceed L2 (126 MB).
  e2e   : keys/s of mgs_sort_host (TanasicSort with one GPU: pinned host
          buffer, H2D + sort + D2H inside the timed call), wall-clock.
  roofline: the onesweep pass kernel, algorithmic bytes (read + write of the
          keys) per launch over its CUDA-event time, against the measured HBM
          copy bandwidth.
  cpu_baseline: the reference's CPU sort (the gnu_parallel branch of
          src/sort_benchmark.cu:103-108, compiled from the reference sources
          into oracle/_ref) on the same 2^30 keys, a few runs bounded by a
          time budget, rank 0 at N=1 only.
With torchrun (N>1) every rank sorts its own 2^30 keys on its own GPU (the path
shards into independent partitions; no data-path collective): weak scaling,
value = all ranks' keys / the slowest rank's time.

--impl reference times the reference's CPU implementation of the path (same
metric, the whole 2^30-key workload per step, keys from the reference's own
DataGenerator) on all host threads, rank 0 only; beside it, for context, the
reference's GPU path (TanasicSort with one GPU, and the CUB sort thrust::sort
dispatches to) on the same keys.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
N_KEYS = 1 << 30
SEED = 2147483647
METRIC = "sorted keys/s (2^30 uint32, plain single-GPU sort)"
WORKLOAD = "plain single-GPU sort: 2^30 uint32 keys, reference DataGenerator 'uniform' [0,2^32), seed 2147483647"


def load_mgs():
    import importlib.util
    spec = importlib.util.spec_from_file_location("mgs", os.path.join(ROOT, "multi-gpu-sorting_b200", "mgs.py"))
    mod = importlib.util.module_from_spec(spec)
    sys.modules["mgs"] = mod
    spec.loader.exec_module(mod)
    return mod


def load_oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    return oracle


def measured_hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        return float(json.load(open(p))["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(kernel: str):
    """DRAM bytes per launch of `kernel` from the committed ncu summary, if any."""
    p = os.path.join(ROOT, "profiles", "radix_onesweep_u32.md")
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("traffic_bytes_per_full_launch:"):
            return float(line.split(":", 1)[1].strip())
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc is not None:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in getattr(self, "lines", []):
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for name, val in zip(names, parts[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        loaded = [s for s in sm if s > 0.5 * (mx or max(sm))] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def max_over_ranks(dist, world: int, value: float, device) -> float:
    """The job's time: the slowest rank's value (all-reduce MAX); with one rank, the value itself."""
    if world <= 1:
        return value
    import torch
    t = torch.tensor([value], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_keys_per_s(world: int, keys_per_rank: int, steps: int, seconds: float) -> float:
    """Whole-job throughput: every rank's keys over the slowest rank's time (weak scaling)."""
    return world * keys_per_rank * steps / seconds


def zipf_segment_offsets(rng, nseg=100_000, total=1 << 28, s=1.2, max_len=1 << 22):
    """Batched workload: nseg segments with Zipf(s) lengths in [1, max_len], rescaled to about `total`
    keys (floor, at least 1 key), in random order."""
    lengths = np.minimum(rng.zipf(s, nseg), max_len).astype(np.float64)
    lengths = np.maximum(1, np.floor(lengths * (total / lengths.sum()))).astype(np.int64)
    rng.shuffle(lengths)
    offs = np.zeros(nseg + 1, dtype=np.int64)
    offs[1:] = np.cumsum(lengths)
    return offs


def verify_segmented(torch, out, src, d_offs, dtype):
    """On the device (4-byte keys): out equals src with every segment [offs[s], offs[s+1]) stably sorted on
    its own, in the sort's order (floats: -0.0 equal to +0.0, NaN by transformed bits). torch sorts (segment,
    order key) pairs stably and gathers the input bits in that order: the expected output, compared byte for
    byte."""
    lens = (d_offs[1:] - d_offs[:-1]).to(torch.int64)
    seg = torch.repeat_interleave(torch.arange(lens.numel(), device=out.device, dtype=torch.int64), lens)
    key = order_key(torch, src, dtype)
    if dtype == "i32":  # signed order key: shift it into [0, 2^32)
        key = key + (1 << 31)
    comp = (seg << 32) | key
    del seg, key
    idx = torch.sort(comp, stable=True)[1]
    del comp
    same = bool(torch.equal(src[idx], out))
    del idx
    torch.cuda.empty_cache()
    return same


def batched_bench(mgs, torch, ctx, dtype="u32", with_plain=True):
    """One segmented-sort call over 10^5 Zipf(1.2) segments (~2^28 keys, uint32 or float32 with -0.0 and NaN)
    against the plain form, one mgs_sort_device launch sequence per segment, on the same device-resident
    keys. The direct call's output is checked on the device (verify_segmented)."""
    rng = np.random.default_rng(11)
    offs = zipf_segment_offsets(rng)
    n = int(offs[-1])
    keys = mgs.generate(dtype, "full-uniform" + ("-specials" if dtype == "f32" else ""), 5, n)
    pristine = torch.from_numpy(keys.view(np.int32)).cuda()
    work = torch.empty_like(pristine)
    d_offs = torch.from_numpy(offs).cuda()
    temp_bytes = mgs.Context.segmented_sort_temp_bytes(dtype, n, offs.size - 1)
    temp = torch.empty(temp_bytes, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    times = []
    for i in range(4):
        with torch.cuda.stream(stream):
            work.copy_(pristine)
            ev[0].record(stream)
            ctx.segmented_sort_device(work.data_ptr(), n, d_offs.data_ptr(), offs.size - 1, dtype, temp.data_ptr(),
                                      temp_bytes, stream.cuda_stream)
            ev[1].record(stream)
        stream.synchronize()
        if i > 0:
            times.append(ev[0].elapsed_time(ev[1]))
    ctx.synchronize()
    batched_ms = statistics.median(times)
    verified = verify_segmented(torch, work, pristine, d_offs, dtype)
    direct_result = work.clone()
    # one more call with the library's per-launch CUDA events on, outside the timed runs: time per kernel
    ctx.set_profiling(True)
    ctx.kernel_times()  # clear
    with torch.cuda.stream(stream):
        work.copy_(pristine)
        ctx.segmented_sort_device(work.data_ptr(), n, d_offs.data_ptr(), offs.size - 1, dtype, temp.data_ptr(),
                                  temp_bytes, stream.cuda_stream)
    stream.synchronize()
    kernel_ms = {name: {"launches": c, "total_ms": t} for name, (c, t) in ctx.kernel_times().items()}
    ctx.set_profiling(False)
    # the same launches recorded once into a CUDA graph (mgs_plan_segmented_create) and replayed
    graph_ms, graph_same = replay_ms(ctx, torch, stream, work, pristine, direct_result,
                                     lambda: ctx.plan_segmented(work.data_ptr(), n, d_offs.data_ptr(), offs.size - 1,
                                                                dtype, temp.data_ptr(), temp_bytes), reps=3)
    del direct_result
    lens = np.diff(offs)
    out = {"segments": int(offs.size - 1), "keys": n, "dtype": dtype,
           "values": "uniform over the full range" + (", 0.1% -0.0 and 0.1% NaN" if dtype == "f32" else ""),
           "lengths": "Zipf(1.2) in [1, 2^22] rescaled to ~2^28 keys, random order",
           "segments_warp_le_1024": int((lens <= 1024).sum()),
           "segments_cta_le_16384": int(((lens > 1024) & (lens <= 16384)).sum()),
           "segments_onesweep_gt_16384": int((lens > 16384).sum()),
           "batched_ms": batched_ms, "batched_keys_per_s": n / (batched_ms / 1e3), "verified": verified,
           "graph_ms": graph_ms, "graph_same_result": graph_same, "kernel_ms": kernel_ms}
    if with_plain:
        out["small_batch"] = small_batch_bench(mgs, torch, ctx, stream)
        # plain form: one sort launch sequence per segment, same stream
        plain_temp = mgs.Context.sort_temp_bytes(dtype, int(np.diff(offs).max()))
        ptemp = torch.empty(plain_temp, dtype=torch.uint8, device="cuda")
        base = work.data_ptr()
        with torch.cuda.stream(stream):
            work.copy_(pristine)
            ev[0].record(stream)
            for s in range(offs.size - 1):
                length = int(offs[s + 1] - offs[s])
                if length > 1:
                    ctx.sort_device(base + 4 * int(offs[s]), length, dtype, ptemp.data_ptr(), plain_temp,
                                    stream.cuda_stream)
            ev[1].record(stream)
        stream.synchronize()
        ctx.synchronize()
        plain_ms = ev[0].elapsed_time(ev[1])
        out.update({"plain_ms": plain_ms, "plain_keys_per_s": n / (plain_ms / 1e3),
                    "speedup_vs_plain": plain_ms / batched_ms})
        del ptemp
    del work, pristine, temp, d_offs
    torch.cuda.empty_cache()
    return out


def replay_ms(ctx, torch, stream, work, pristine, expected, make_plan, reps):
    """Median CUDA-event time of `reps` replays of a recorded plan (input restored before each, outside the
    timed region) and whether the last replay's result equals `expected`."""
    plan = make_plan()
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    times = []
    try:
        for i in range(reps + 1):
            with torch.cuda.stream(stream):
                work.copy_(pristine)
                ev[0].record(stream)
                plan.launch(stream.cuda_stream)
                ev[1].record(stream)
            stream.synchronize()
            if i > 0:
                times.append(ev[0].elapsed_time(ev[1]))
        ctx.synchronize()
        same = bool(torch.equal(work, expected))
    finally:
        plan.close()
    return statistics.median(times), same


def small_batch_bench(mgs, torch, ctx, stream, reps=20):
    """A small batch (1024 Zipf(1.2) segments, 2^18 u32 keys) where launch overhead matters: the direct
    segmented call against its recorded CUDA graph, median CUDA-event time per call."""
    rng = np.random.default_rng(12)
    offs = zipf_segment_offsets(rng, nseg=1024, total=1 << 18, max_len=1 << 14)
    n = int(offs[-1])
    pristine = torch.from_numpy(mgs.generate("u32", "full-uniform", 6, n).view(np.int32)).cuda()
    work = torch.empty_like(pristine)
    d_offs = torch.from_numpy(offs).cuda()
    temp_bytes = mgs.Context.segmented_sort_temp_bytes("u32", n, offs.size - 1)
    temp = torch.empty(temp_bytes, dtype=torch.uint8, device="cuda")
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
    times = []
    for i in range(reps + 1):
        with torch.cuda.stream(stream):
            work.copy_(pristine)
            ev[0].record(stream)
            ctx.segmented_sort_device(work.data_ptr(), n, d_offs.data_ptr(), offs.size - 1, "u32", temp.data_ptr(),
                                      temp_bytes, stream.cuda_stream)
            ev[1].record(stream)
        stream.synchronize()
        if i > 0:
            times.append(ev[0].elapsed_time(ev[1]))
    ctx.synchronize()
    direct_ms = statistics.median(times)
    expected = work.clone()
    graph_ms, same = replay_ms(ctx, torch, stream, work, pristine, expected,
                               lambda: ctx.plan_segmented(work.data_ptr(), n, d_offs.data_ptr(), offs.size - 1, "u32",
                                                          temp.data_ptr(), temp_bytes), reps)
    return {"segments": int(offs.size - 1), "keys": n, "direct_ms": direct_ms, "graph_ms": graph_ms,
            "graph_same_result": same}


def served_bench(mgs, torch, budget_s=2.0):
    """Batched and served sorting, request stream: Poisson arrivals at 10/50/90% of the plain form's measured
    peak (and the served form at 90% of its own), key type uniform over u32/i32/f32/u64, request keys resident
    in HBM (mgs_server_submit_device, sorted in place). Two size mixes: log-uniform over 2^10..2^26 keys, and
    small requests only (2^10..2^18). Forms: plain = one request per launch sequence, one at a time
    (num_slots 1, no coalescing); served = continuous batching (4 batches in flight, requests up to 2^20 keys
    coalesced, admission by free pool memory). Peak: the whole pool of 96 requests submitted at once (a full
    queue), four rounds, keys over the server's busy time. Every request sorts fresh keys: once a request
    finishes, its buffer is restored from a pristine device copy (outside its latency) before it is submitted
    again."""
    import threading
    import queue as _queue
    types = ["u32", "i32", "f32", "u64"]
    out = {"arrivals": "Poisson", "types": types, "requests": "device-resident (mgs_server_submit_device)",
           "offered_load": "fraction of the plain form's peak keys/s (served also at 0.9 of its own peak)",
           "input": "each request's keys restored from a pristine device copy after it completes"}
    for mix, (lo, hi) in (("log-uniform 2^10..2^26", (10, 26)), ("log-uniform 2^10..2^18", (10, 18))):
        rng = np.random.default_rng(7)
        pool = []
        for i, n in enumerate((2 ** rng.uniform(lo, hi, 96)).astype(np.int64)):
            dt = types[i % 4]
            a = mgs.generate(dt, "full-uniform" + ("-specials" if dt == "f32" else ""), 100 + i, int(n))
            st = np.int32 if a.dtype.itemsize == 4 else np.int64
            pristine = torch.from_numpy(a.view(st)).cuda()
            pool.append((dt, int(n), pristine, pristine.clone()))
        torch.cuda.synchronize()
        mean_keys = float(np.mean([p[1] for p in pool]))
        restore_stream = torch.cuda.Stream()

        def restore(idx):
            with torch.cuda.stream(restore_stream):
                torch._foreach_copy_([pool[i][3] for i in idx], [pool[i][2] for i in idx])
            restore_stream.synchronize()

        def summary(st):
            return {"requests": st["completed"], "keys_per_s": st["keys"] / max(st["busy_s"], 1e-9),
                    "p50_ms": st["p50_us"] / 1e3, "p99_ms": st["p99_us"] / 1e3, "batches": st["batches"],
                    "kernel_launches": st["kernel_launches"]}

        def burst(srv, rounds):
            """The whole pool submitted at once, `rounds` times (inputs restored between rounds, outside the
            server's busy time): the server's throughput with a full queue."""
            keys = busy = 0.0
            lat = []
            batches = launches = 0
            for _ in range(rounds):
                restore(range(len(pool)))
                srv.stats(reset=True)
                ids = [srv.submit_device(w.data_ptr(), n, dt) for dt, n, _, w in pool]
                assert all(srv.wait(i) == mgs.MGS_OK for i in ids)
                st = srv.stats()
                keys += st["keys"]
                busy += st["busy_s"]
                lat += [st["p50_us"], st["p99_us"]]
                batches += st["batches"]
                launches += st["kernel_launches"]
            restore(range(len(pool)))
            return {"requests": rounds * len(pool), "keys_per_s": keys / max(busy, 1e-9), "rounds": rounds,
                    "p50_ms_median_round": statistics.median(lat[0::2]) / 1e3,
                    "p99_ms_median_round": statistics.median(lat[1::2]) / 1e3, "batches": batches,
                    "kernel_launches": launches}

        def run(srv, rate, duration, max_requests):
            """Poisson arrivals at `rate` requests/s; a finished request's buffer is restored (in groups, on a
            side stream) before it is submitted again."""
            free = _queue.Queue()
            for i in range(len(pool)):
                free.put(i)
            done = _queue.Queue()

            def reaper():
                stop = False
                while not stop:
                    items = [done.get()]
                    while True:
                        try:
                            items.append(done.get_nowait())
                        except _queue.Empty:
                            break
                    if items[-1] is None:
                        stop = True
                        items.pop()
                    for rid, _ in items:
                        assert srv.wait(rid) == mgs.MGS_OK
                    if items:
                        restore([i for _, i in items])
                        for _, i in items:
                            free.put(i)

            th = threading.Thread(target=reaper)
            th.start()
            srv.stats(reset=True)
            t0 = time.perf_counter()
            nxt = t0
            sent = 0
            while sent < max_requests and time.perf_counter() - t0 < duration:
                nxt += rng.exponential(1.0 / rate)
                while time.perf_counter() < nxt:
                    pass
                i = free.get()
                dt, n, _, work = pool[i]
                done.put((srv.submit_device(work.data_ptr(), n, dt), i))
                sent += 1
            done.put(None)
            th.join()
            return summary(srv.stats())

        res = {"pool": len(pool), "mean_request_keys": mean_keys}
        forms = [("plain", dict(num_slots=1, coalesce_keys=0)),
                 ("served", dict(num_slots=4, coalesce_keys=1 << 20))]
        plain_peak = None
        for name, cfg in forms:
            srv = mgs.Server(0, **cfg)
            try:
                burst(srv, 1)  # warm-up
                peak = burst(srv, 4)
                if plain_peak is None:
                    plain_peak = peak["keys_per_s"]
                levels = []
                targets = [(load, load * plain_peak) for load in (0.1, 0.5, 0.9)]
                if name == "served":
                    targets.append((round(0.9 * peak["keys_per_s"] / plain_peak, 3), 0.9 * peak["keys_per_s"]))
                for load, keys_per_s in targets:
                    r = run(srv, keys_per_s / mean_keys, budget_s, 20_000)
                    r["offered_load"] = load
                    r["offered_keys_per_s"] = keys_per_s
                    levels.append(r)
                res[name] = {"peak": peak, "loads": levels, "config": cfg}
            finally:
                srv.close()
        res["served_over_plain_peak"] = res["served"]["peak"]["keys_per_s"] / res["plain"]["peak"]["keys_per_s"]
        out[mix] = res
        del pool
        torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------- sweeps ----
# `bench.py --sweep types|merge|ooc` measures the other workloads of the sort
# API on one GPU and prints one JSON line per case instead of the headline line.

SWEEP_DISTS = ["full-uniform", "normal0", "zipf", "sorted-full", "reverse-sorted-full", "nearly-sorted-swaps",
               "all-equal"]


def order_key(torch, t, dtype):
    """int64 tensor whose signed order is the sort's order of the keys in t (same bits, int32/int64 storage):
    unsigned for u32/u64, two's complement for i32, and for f32 the radix order (-0.0 equal to +0.0, NaN by
    transformed bits)."""
    if dtype == "u32":
        return t.to(torch.int64) & 0xFFFFFFFF
    if dtype == "i32":
        return t.to(torch.int64)
    if dtype == "u64":
        return t ^ (-(1 << 63))
    u = t.to(torch.int64) & 0xFFFFFFFF
    u = torch.where(u == 0x80000000, torch.zeros_like(u), u)  # -0.0 -> +0.0
    return torch.where(u >= 0x80000000, 0xFFFFFFFF - u, u + 0x80000000)


def same_multiset_invariants(torch, a, b, dtype):
    """Multiset invariants of two key tensors: sum and sum of squares (mod 2^64), the sum of a
    multiplicative hash of every key (mod 2^64), and a 2^16-bin histogram of the order key's top bits."""
    shift = 16 if a.element_size() == 4 else 48

    def inv(t):
        x = t.to(torch.int64)
        h = x * -7046029254386353131  # 0x9E3779B97F4A7C15 as a signed 64-bit constant
        top = (order_key(torch, t, dtype) >> shift) & 0xFFFF
        return [x.sum(), (x * x).sum(), (h ^ (h >> 29)).sum(), torch.bincount(top, minlength=1 << 16)]

    return all(torch.equal(u, v) for u, v in zip(inv(a), inv(b)))


def verify_sorted_permutation(torch, out, src, dtype):
    """On the device: out is ascending in the sort's order, holds the same multiset of bit patterns as src,
    and (floats) keeps the input order of -0.0 and +0.0, which compare equal. Together these fix every
    output byte."""
    k = order_key(torch, out, dtype)
    if not bool((k[1:] >= k[:-1]).all()):
        return False
    if out.numel() < (1 << 31) - 1:
        if not torch.equal(torch.sort(out.view(-1))[0], torch.sort(src.view(-1))[0]):
            return False
    elif not same_multiset_invariants(torch, out, src, dtype):  # beyond torch.sort's element limit
        return False
    if dtype == "f32":
        bits_in = src.to(torch.int64) & 0xFFFFFFFF
        bits_out = out.to(torch.int64) & 0xFFFFFFFF
        z_in = bits_in[(bits_in == 0) | (bits_in == 0x80000000)]
        z_out = bits_out[(bits_out == 0) | (bits_out == 0x80000000)]
        if not torch.equal(z_in, z_out):
            return False
    return True


def sweep_types(mgs, torch, n, reps=3):
    """Plain device sort of n keys of u32, i32, f32 and u64 over seven distributions (float arrays carry 0.1%
    -0.0 and 0.1% NaN): keys/s and the fraction of the HBM roofline for the canonical n*w*(2P+1) bytes."""
    ctx = mgs.Context(0)
    peak, _ = measured_hbm_peak()
    stream = torch.cuda.Stream()
    for dtype in ["u32", "i32", "f32", "u64"]:
        w = 8 if dtype == "u64" else 4
        storage = (np.int64, torch.int64) if w == 8 else (np.int32, torch.int32)
        temp_bytes = mgs.Context.sort_temp_bytes(dtype, n)
        temp = torch.empty(temp_bytes, dtype=torch.uint8, device="cuda")
        for dist in SWEEP_DISTS:
            name = dist + ("-specials" if dtype == "f32" else "")
            src = torch.empty(n, dtype=storage[1], device="cuda")
            if dist == "normal0":  # log / cos of the host C library: generated on the host
                src.copy_(torch.from_numpy(mgs.generate(dtype, name, SEED, n).view(storage[0])))
            else:  # the same bytes, generated in place on the device
                ctx.generate_device(src.data_ptr(), n, dtype, name, SEED)
            work = torch.empty_like(src)
            times = []
            for i in range(reps + 1):
                with torch.cuda.stream(stream):
                    work.copy_(src)
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    ctx.sort_device(work.data_ptr(), n, dtype, temp.data_ptr(), temp_bytes, stream.cuda_stream)
                    b.record(stream)
                stream.synchronize()
                if i > 0:
                    times.append(a.elapsed_time(b))
            ok = verify_sorted_permutation(torch, work, src, dtype)
            ms = statistics.median(times)
            alg = n * w * (2 * w + 1)
            print(json.dumps({"sweep": "types", "dtype": dtype, "distribution": name, "n": n, "ms": ms,
                              "keys_per_s": n / (ms / 1e3), "hbm_alg_gbs": alg / (ms / 1e3) / 1e9,
                              "roofline_frac": alg / (ms / 1e3) / 1e9 / peak, "reps": reps, "verified": ok}),
                  flush=True)
            del src, work
        del temp
    ctx.close()


def sweep_generate(mgs, torch, n):
    """Input generation of n keys on the device (mgs_generate_device) against the host generator (mgs_generate,
    all host threads) producing the same bytes: wall-clock seconds of each call and whether the bytes agree."""
    ctx = mgs.Context(0)
    cases = [("u32", "uniform"), ("u32", "full-uniform"), ("u32", "zipf"), ("u32", "sorted"), ("u32", "staggered"),
             ("f32", "nearly-sorted-swaps-specials"), ("u64", "full-uniform"), ("f64", "bucket-sorted")]
    for dtype, dist in cases:
        dt = mgs.np_dtype(dtype)
        st_np, st_t = (np.int32, torch.int32) if dt.itemsize == 4 else (np.int64, torch.int64)
        d = torch.empty(n, dtype=st_t, device="cuda")
        ctx.generate_device(d.data_ptr(), min(n, 1 << 20), dtype, dist, SEED)  # loads the kernels
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        ctx.generate_device(d.data_ptr(), n, dtype, dist, SEED)
        dev_s = time.perf_counter() - t0
        h = mgs.host_empty(n, dt)
        t0 = time.perf_counter()
        mgs.generate(dtype, dist, SEED, n, out=h)
        host_s = time.perf_counter() - t0
        same = bool(torch.equal(d, torch.from_numpy(h.view(st_np)).cuda()))
        print(json.dumps({"sweep": "generate", "dtype": dtype, "distribution": dist, "n": n, "device_s": dev_s,
                          "host_s": host_s, "host_threads": os.cpu_count(), "speedup": host_s / dev_s,
                          "bytes_identical": same}), flush=True)
        del d, h
    ctx.close()


def dirichlet_lengths(rng, k, total):
    w = rng.dirichlet(np.ones(k))
    lens = np.floor(w * total).astype(np.int64)
    lens[np.argmax(lens)] += total - int(lens.sum())
    return [int(x) for x in lens]


def sweep_merge(mgs, torch, n, reps=3):
    """Chunked merge path (TanasicSort over g chunks of one GPU, g in 2, 4, 8) and the k-way merge of k in
    2, 8, 16, 32, 64 sorted runs with Dirichlet(1) lengths, n uint32 keys each."""
    ctx = mgs.Context(0)
    peak, _ = measured_hbm_peak()
    g = torch.Generator(device="cuda")
    g.manual_seed(SEED)
    src = torch.randint(-2 ** 31, 2 ** 31 - 1, (n,), dtype=torch.int32, device="cuda", generator=g)
    work = torch.empty_like(src)
    for chunks in (2, 4, 8):
        times = []
        for i in range(reps + 1):
            work.copy_(src)
            torch.cuda.synchronize()
            ctx.set_profiling(i > 0)
            t0 = time.perf_counter()
            ctx.tanasic_sort_device(work.data_ptr(), n, "u32", chunks)
            dt = time.perf_counter() - t0
            if i > 0:
                times.append(dt)
        kt = ctx.kernel_times()
        ctx.set_profiling(False)
        ok = verify_sorted_permutation(torch, work, src, "u32")
        s = statistics.median(times)
        merge_ms = sum(v[1] for k_, v in kt.items() if not k_.startswith("radix")) / reps
        sort_ms = sum(v[1] for k_, v in kt.items() if k_.startswith("radix")) / reps
        print(json.dumps({"sweep": "chunked_merge", "dtype": "u32", "n": n, "chunks": chunks, "s": s,
                          "keys_per_s": n / s, "chunk_sort_kernel_ms": sort_ms, "merge_kernel_ms": merge_ms,
                          "kernels": {k_: {"launches": v[0] // reps, "ms": v[1] / reps} for k_, v in kt.items()},
                          "verified": ok}), flush=True)
    del work
    rng = np.random.default_rng(SEED)
    out = torch.empty_like(src)
    orc = None
    for k in (2, 8, 16, 32, 64):
        lens = dirichlet_lengths(rng, k, n)
        offs = np.concatenate([[0], np.cumsum(lens)])
        runs = src.clone()
        for r in range(k):
            if lens[r] > 1:
                ctx.sort_device(runs.data_ptr() + 4 * int(offs[r]), lens[r], "u32")
        ctx.synchronize()
        ptrs = [runs.data_ptr() + 4 * int(offs[r]) for r in range(k)]
        temp_bytes = mgs.Context.merge_temp_bytes("u32", k, n)
        temp = torch.empty(max(temp_bytes, 1), dtype=torch.uint8, device="cuda")
        stream = torch.cuda.Stream()
        times = []
        for i in range(reps + 1):
            ctx.set_profiling(i > 0)
            with torch.cuda.stream(stream):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                ctx.kway_merge_device(ptrs, lens, out.data_ptr(), "u32", temp.data_ptr(), temp_bytes,
                                      stream.cuda_stream)
                b.record(stream)
            stream.synchronize()
            if i > 0:
                times.append(a.elapsed_time(b))
        kt = ctx.kernel_times()
        ctx.set_profiling(False)
        ok = verify_sorted_permutation(torch, out, src, "u32")
        ms = statistics.median(times)
        alg = 2 * 4 * n
        line = {"sweep": "kway_merge", "dtype": "u32", "n": n, "k": k, "run_lengths": "Dirichlet(1)", "ms": ms,
                "keys_per_s": n / (ms / 1e3), "hbm_alg_gbs": alg / (ms / 1e3) / 1e9,
                "roofline_frac": alg / (ms / 1e3) / 1e9 / peak, "verified": ok,
                "kernels": {k_: {"launches": v[0] // reps, "ms": v[1] / reps} for k_, v in kt.items()}}
        # cpu_baseline: the reference's own CPU merge (__gnu_parallel::multiway_merge through oracle/_ref)
        # on a bounded sample: the first 2^27 keys split into k runs of the same proportions.
        if orc is None:
            orc = load_oracle()
        if orc.ref_available():
            m = 1 << 27
            sl = [max(1, int(x * m / n)) for x in lens]
            host_runs = []
            hsrc = src[: sum(sl)].cpu().numpy().view(np.uint32)
            o = 0
            for x in sl:
                host_runs.append(np.sort(hsrc[o:o + x]))
                o += x
            threads = os.cpu_count() or 1
            t0 = time.perf_counter()
            orc.ref_multiway_merge(host_runs, threads)
            dt = time.perf_counter() - t0
            line["cpu_baseline"] = {"value": sum(sl) / dt, "unit": "keys/s", "cores": threads, "kind": "reference",
                                    "sample": f"{sum(sl)} keys in {k} runs of the same proportions "
                                              "(__gnu_parallel::multiway_merge, src/gowanlock_sort.cuh:73-74)"}
        print(json.dumps(line), flush=True)
        del runs, temp
    ctx.close()


def sweep_range(mgs, torch, n=1 << 30, reps=3):
    """Descending order and bit ranges (CUB's SortKeysDescending / begin_bit, end_bit forms) on 2^30 device-
    resident u32 keys: descending over all 32 bits, and ascending / descending by bits [8, 24). Checked on the
    device against torch's stable sort of the same bit field. Algorithmic bytes: 2 x 4 B per pass that the range
    needs plus one histogram read."""
    ctx = mgs.Context(0)
    peak, _ = measured_hbm_peak()
    stream = torch.cuda.Stream()
    src = torch.empty(n, dtype=torch.int32, device="cuda")
    ctx.generate_device(src.data_ptr(), n, "u32", "full-uniform", SEED)
    work = torch.empty_like(src)
    temp_bytes = mgs.Context.sort_temp_bytes("u32", n)
    temp = torch.empty(temp_bytes, dtype=torch.uint8, device="cuda")
    for begin, end, desc in ((0, 32, True), (8, 24, False), (8, 24, True)):
        times = []
        for i in range(reps + 1):
            with torch.cuda.stream(stream):
                work.copy_(src)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                ctx.sort_range_device(work.data_ptr(), n, "u32", begin, end, desc, d_temp=temp.data_ptr(),
                                      temp_bytes=temp_bytes, stream=stream.cuda_stream)
                b.record(stream)
            stream.synchronize()
            if i > 0:
                times.append(a.elapsed_time(b))
        ctx.synchronize()
        field = ((src.to(torch.int64) & 0xFFFFFFFF) >> begin) & ((1 << (end - begin)) - 1)
        if desc:
            field = ((1 << (end - begin)) - 1) - field
        idx = torch.sort(field, stable=True)[1]
        del field
        ok = bool(torch.equal(src[idx], work))
        del idx
        torch.cuda.empty_cache()
        ms = statistics.median(times)
        passes = (end - begin + 7) // 8
        alg = n * 4 * (2 * passes + 1)
        print(json.dumps({"sweep": "range", "dtype": "u32", "n": n, "begin_bit": begin, "end_bit": end,
                          "descending": desc, "ms": ms, "keys_per_s": n / (ms / 1e3),
                          "hbm_alg_gbs": alg / (ms / 1e3) / 1e9, "roofline_frac": alg / (ms / 1e3) / 1e9 / peak,
                          "reps": reps, "verified": ok}), flush=True)
    ctx.close()


def sweep_pairs(mgs, torch, n32=1 << 30, reps=3):
    """Key-value sort (thrust::sort_by_key order) on device-resident data: 2^30 u32 keys with u32 values and 2^29
    u64 keys with u64 values; the values are the input positions, so the result is checked by gathering the input
    through them (ascending, a permutation, equal keys in input order). Algorithmic bytes: every pass reads and
    writes keys and values, plus one histogram read of the keys."""
    ctx = mgs.Context(0)
    peak, _ = measured_hbm_peak()
    stream = torch.cuda.Stream()
    for dtype, n, vb in (("u32", n32, 4), ("u64", n32 // 2, 8)):
        w = 4 if dtype == "u32" else 8
        st = torch.int32 if w == 4 else torch.int64
        vt = torch.int32 if vb == 4 else torch.int64
        src = torch.from_numpy(mgs.generate(dtype, "full-uniform", SEED, n).view(np.int32 if w == 4 else np.int64)).cuda()
        keys, vals = torch.empty_like(src), torch.empty(n, dtype=vt, device="cuda")
        iota = torch.arange(n, dtype=vt, device="cuda")
        temp_bytes = mgs.Context.sort_pairs_temp_bytes(dtype, vb, n)
        temp = torch.empty(temp_bytes, dtype=torch.uint8, device="cuda")
        times = []
        for i in range(reps + 1):
            with torch.cuda.stream(stream):
                keys.copy_(src)
                vals.copy_(iota)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                ctx.sort_pairs_device(keys.data_ptr(), vals.data_ptr(), vb, n, dtype, temp.data_ptr(), temp_bytes,
                                      stream.cuda_stream)
                b.record(stream)
            stream.synchronize()
            if i > 0:
                times.append(a.elapsed_time(b))
        ctx.synchronize()
        idx = vals.to(torch.int64)
        k = order_key(torch, keys, dtype)
        ok = bool(torch.equal(src[idx], keys)) and bool((k[1:] >= k[:-1]).all())
        same = k[1:] == k[:-1]
        ok = ok and bool((idx[1:][same] > idx[:-1][same]).all())
        ok = ok and bool(torch.equal(torch.sort(idx)[0], torch.arange(n, device="cuda")))
        ms = statistics.median(times)
        alg = n * (2 * w * (w + vb) + w)
        print(json.dumps({"sweep": "pairs", "dtype": dtype, "value_bytes": vb, "n": n, "ms": ms,
                          "pairs_per_s": n / (ms / 1e3), "hbm_alg_gbs": alg / (ms / 1e3) / 1e9,
                          "roofline_frac": alg / (ms / 1e3) / 1e9 / peak, "verified": ok}), flush=True)
        del src, keys, vals, iota, temp, idx, k, same
    ctx.close()


def sweep_tune(mgs, out_path, max_n=1 << 28, reps=3):
    """Autotuner run: every onesweep variant (7 tile shapes x 2 ranking modes) timed per size class up to max_n
    for 4- and 8-byte keys; the fastest per class goes into the table, which is written to out_path if given."""
    ctx = mgs.Context(0)
    for dtype in ("u32", "u64"):
        for smp in ctx.autotune(dtype, max_n, reps):
            print(json.dumps({"sweep": "tune", "dtype": dtype, **smp}), flush=True)
    if out_path:
        mgs.tune_save(out_path)
    ctx.close()


def link_bandwidth(torch, nbytes=1 << 32):
    """Pinned host<->device copy bandwidth (GB/s): H2D alone, D2H alone, and both at once (full duplex)."""
    h_in = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    h_out = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    d_a = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    d_b = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()

    def timed(fn):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        return time.perf_counter() - t0

    def h2d():
        with torch.cuda.stream(s1):
            d_a.copy_(h_in, non_blocking=True)

    def d2h():
        with torch.cuda.stream(s2):
            h_out.copy_(d_b, non_blocking=True)

    def both():
        h2d()
        d2h()

    h2d(), d2h()
    t_h2d, t_d2h, t_both = timed(h2d), timed(d2h), timed(both)
    return {"h2d_gbs": nbytes / t_h2d / 1e9, "d2h_gbs": nbytes / t_d2h / 1e9,
            "duplex_gbs_each": nbytes / t_both / 1e9, "bytes": nbytes}


def sweep_ooc(mgs, torch, n, chunk=1 << 28):
    """Out-of-core GowanlockSort pipeline over n uint64 keys in pinned host memory, chunks of `chunk` keys,
    with the GPU k-way merge and with the reference's CPU multiway merge; end-to-end keys/s against the
    host-link bound (every key crosses the link twice per direction with the GPU merge, once with the CPU
    merge)."""
    link = link_bandwidth(torch)
    print(json.dumps({"sweep": "link", **link}), flush=True)
    ctx = mgs.Context(0)
    h = mgs.host_empty(n, np.uint64)
    for merge_on_gpu in (True, False):
        mgs.generate("u64", "full-uniform", SEED, n, out=h)
        x0 = int(np.bitwise_xor.reduce(h))
        s0 = int(h.sum(dtype=np.uint64))
        t0 = time.perf_counter()
        ctx.gowanlock_sort(h, chunk_size=chunk, merge_group_size=0, num_buffers=3, merge_on_gpu=merge_on_gpu)
        dt = time.perf_counter() - t0
        phases = {p: ctx.phase_seconds(p) for p in ("memory_allocation", "sort_phase", "merge_phase")}
        ok = True
        step = 1 << 28
        for o in range(0, n, step):
            seg = h[o:min(n, o + step + 1)]
            if not bool(np.all(seg[1:] >= seg[:-1])):
                ok = False
                break
        ok = ok and int(np.bitwise_xor.reduce(h)) == x0 and int(h.sum(dtype=np.uint64)) == s0
        w = 8
        crossings = 2 if merge_on_gpu else 1
        bound_s = crossings * n * w / (min(link["duplex_gbs_each"], link["h2d_gbs"], link["d2h_gbs"]) * 1e9)
        print(json.dumps({"sweep": "out_of_core", "dtype": "u64", "n": n, "bytes": n * w, "chunk": chunk,
                          "num_buffers": 3, "merge": "gpu" if merge_on_gpu else "cpu (reference multiway_merge)",
                          "s": dt, "keys_per_s": n / dt, "phases_s": phases,
                          "link_bound_s": bound_s, "link_frac": bound_s / dt, "verified": ok}), flush=True)
    ctx.close()


def cpu_reference_sort(orc, base: np.ndarray, budget_s: float, max_reps: int):
    """Times the reference's gnu_parallel sort on copies of `base` (bounded)."""
    threads = orc.ref_num_procs()
    work = np.empty_like(base)
    times = []
    t_end = time.perf_counter() + budget_s
    for _ in range(max_reps):
        np.copyto(work, base)
        times.append(orc.ref_gnu_parallel_sort(work, threads))
        if time.perf_counter() > t_end:
            break
    return base.size / statistics.median(times), threads, times


def reference_gpu_path(orc, base: np.ndarray, reps: int = 2):
    """The reference's own GPU path on the same keys, for context beside the CPU arm: TanasicSort<T> with
    one GPU (src/tanasic_sort.cuh:223-299: H2D, thrust::sort, D2H; its own sort_phase timer) and the
    device-resident CUB DeviceRadixSort::SortKeys that thrust::sort dispatches to (CUDA events,
    src/local_gpu_sort_algorithm_benchmark.cu:51-67). Both come from oracle/_ref only."""
    import torch
    n = base.size
    phase = []
    work = np.empty_like(base)
    for _ in range(reps):
        np.copyto(work, base)
        orc.ref_tanasic_sort(work, 0)
        phase.append(orc.ref_phase_seconds("sort_phase"))
    ok = bool(np.all(work[1:] >= work[:-1]))
    d_in = torch.from_numpy(base.view(np.int32)).cuda()
    d_out = torch.empty_like(d_in)
    _, need = orc.ref_cub_sort_device_ms(0, d_in.data_ptr(), d_out.data_ptr(), n)
    temp = torch.empty(max(need, 1), dtype=torch.uint8, device="cuda")
    cub_ms = []
    for i in range(reps + 3):  # out of place from the same input: every run sorts the same keys
        torch.cuda.synchronize()
        ms, _ = orc.ref_cub_sort_device_ms(0, d_in.data_ptr(), d_out.data_ptr(), n, temp.data_ptr(), need)
        if i >= 3:
            cub_ms.append(ms)
    del d_in, d_out, temp
    sp = statistics.median(phase)
    cm = statistics.median(cub_ms)
    return {"tanasic_sort_phase_s": sp, "tanasic_keys_per_s": n / sp, "cub_device_ms": cm,
            "cub_device_keys_per_s": n / (cm / 1e3), "reps": reps, "sorted": ok,
            "what": "reference TanasicSort<uint32_t> g=1 (H2D + thrust::sort + D2H, its sort_phase timer) and "
                    "cub::DeviceRadixSort::SortKeys on device-resident keys (CUDA events), same keys"}


def run_reference(args, rank):
    """The reference arm: the reference's own CPU sort (the gnu_parallel branch of src/sort_benchmark.cu:103-108,
    compiled from the reference sources into oracle/_ref) on the full workload, every host thread, rank 0 only.
    The keys come from the reference's own DataGenerator, so nothing of the engine is loaded."""
    if rank != 0:
        return
    orc = load_oracle()
    if not orc.ref_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libref.so not built"}))
        return
    n = args.n
    base = orc.ref_generate(np.uint32, "uniform", SEED, n)
    threads = orc.ref_num_procs()
    work = np.empty_like(base)
    for _ in range(args.warmup):
        np.copyto(work, base)
        orc.ref_gnu_parallel_sort(work, threads)
    times = []
    for _ in range(args.steps):
        np.copyto(work, base)
        times.append(orc.ref_gnu_parallel_sort(work, threads))
    ok = bool(np.all(work[1:] >= work[:-1]))
    del work
    value = n * len(times) / sum(times)
    gpu_path = None
    if not args.no_reference_gpu:
        gpu_path = reference_gpu_path(orc, base)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "keys/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sum(times) / len(times),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (reference DataGenerator, oracle/_ref)",
        "config": {"workload": WORKLOAD, "keys": n, "same_config": n == N_KEYS, "verified_sorted": ok,
                   "algorithm": "reference gnu_parallel sort (src/sort_benchmark.cu:103-108), oracle/_ref"},
        "cpu_baseline": {"value": value, "unit": "keys/s", "cores": threads, "kind": "reference",
                         "sample": f"the whole workload ({n} uint32 keys) per step, {args.steps} steps, "
                                   f"{args.warmup} warm-up steps"},
        "e2e": {"value": value, "unit": "keys/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_gpu_path": gpu_path,
    }
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="mgs", choices=["mgs", "reference"])
    ap.add_argument("--n", type=int, default=N_KEYS)
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batched", action="store_true", help="skip the batched (segmented) measurement")
    ap.add_argument("--no-served", action="store_true", help="skip the serving-loop measurement")
    ap.add_argument("--no-reference-gpu", action="store_true",
                    help="--impl reference: skip timing the reference's GPU path beside its CPU sort")
    ap.add_argument("--sweep", choices=["types", "merge", "ooc", "tune", "pairs", "generate", "range"],
                    help="measure another workload of the sort API instead (one JSON line per case)")
    ap.add_argument("--sweep-n", type=int, default=0, help="keys per case of --sweep (0: the workload's default)")
    ap.add_argument("--tune-out", default="", help="--sweep tune: write the tuned variant table to this file")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))

    if args.impl == "reference":
        run_reference(args, rank)
        return

    if args.sweep:
        import torch
        torch.cuda.set_device(local_rank)
        mgs = load_mgs()
        if args.sweep == "types":
            sweep_types(mgs, torch, args.sweep_n or N_KEYS)
        elif args.sweep == "generate":
            sweep_generate(mgs, torch, args.sweep_n or N_KEYS)
        elif args.sweep == "pairs":
            sweep_pairs(mgs, torch, args.sweep_n or (1 << 30))
        elif args.sweep == "range":
            sweep_range(mgs, torch, args.sweep_n or (1 << 30))
        elif args.sweep == "tune":
            sweep_tune(mgs, args.tune_out, args.sweep_n or (1 << 28))
        elif args.sweep == "merge":
            sweep_merge(mgs, torch, args.sweep_n or (1 << 31))
        else:
            sweep_ooc(mgs, torch, args.sweep_n or (1 << 32))
        return

    import torch
    import torch.distributed as dist
    from datetime import timedelta

    torch.cuda.set_device(local_rank)
    if world > 1:
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local_rank))

    mgs = load_mgs()
    n = args.n
    ctx = mgs.Context(local_rank)
    keys_np = mgs.generate("u32", "uniform", SEED + rank, n)
    pristine = torch.from_numpy(keys_np.view(np.int32)).cuda()
    work = torch.empty_like(pristine)
    temp_bytes = mgs.Context.sort_temp_bytes("u32", n)
    temp = torch.empty(temp_bytes, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream

    def one_sort(timed_events=None):
        with torch.cuda.stream(stream):
            work.copy_(pristine)
            if timed_events is not None:
                timed_events[0].record(stream)
            ctx.sort_device(work.data_ptr(), n, "u32", temp.data_ptr(), temp_bytes, sptr)
            if timed_events is not None:
                timed_events[1].record(stream)

    for _ in range(args.warmup):
        one_sort()
    stream.synchronize()
    ctx.synchronize()

    # verify the warm-up result on the device: ascending and the same multiset of keys as the input (both
    # sorted by torch and compared), which for integer keys fixes every output byte
    ok = verify_sorted_permutation(torch, work, pristine, "u32")
    torch.cuda.empty_cache()

    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.launch_count(reset=True)
    ctx.set_profiling(True)
    ctx.kernel_times()  # clear
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(local_rank) as clocks:
        for i in range(args.steps):
            one_sort(evs[i])
        stream.synchronize()
    torch.cuda.synchronize()
    launches = ctx.launch_count(reset=True)
    ktimes = ctx.kernel_times()
    ctx.set_profiling(False)
    ctx.synchronize()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    ok = ok and verify_sorted_permutation(torch, work, pristine, "u32")  # the last timed step's output
    torch.cuda.empty_cache()
    total_ms = max_over_ranks(dist, world, sum(step_ms), "cuda")
    value = job_keys_per_s(world, n, args.steps, total_ms / 1e3)

    # end to end through the public host API (mgs_sort_host), pinned buffers
    h = mgs.host_empty(n, np.uint32)
    e2e_times = []
    for i in range(args.e2e_steps + 1):
        np.copyto(h, keys_np)
        if world > 1:
            dist.barrier()
        t0 = time.perf_counter()
        ctx.sort_host(h)
        dt = time.perf_counter() - t0
        if i > 0:  # first call warms the arena
            e2e_times.append(dt)
    e2e_ok = bool(np.all(h[1:] >= h[:-1]))
    e2e_s = max_over_ranks(dist, world, sum(e2e_times), "cuda")
    e2e_value = job_keys_per_s(world, n, len(e2e_times), e2e_s) if e2e_times else None

    peak, peak_kind = measured_hbm_peak()
    one = ktimes.get("radix_onesweep", (0, 0.0))
    hist = ktimes.get("radix_histogram", (0, 0.0))
    roof = None
    if one[0] > 0:
        avg_ms = one[1] / one[0]
        alg_bytes = 2 * 4 * n  # each pass reads and writes every key
        achieved = alg_bytes / (avg_ms / 1e3) / 1e9
        traffic = committed_traffic("radix_onesweep") if n == N_KEYS else None
        roof = {"bound": "hbm", "kernel": "radix_onesweep", "achieved": achieved, "peak": peak, "unit": "GB/s",
                "frac": achieved / peak, "peak_kind": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "traffic": traffic, "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms}
    sort_alg_bytes = 36 * n  # 4 passes x (read + write) + one histogram read, 4-byte keys
    sort_ms = total_ms / args.steps

    batched = None
    served = None
    if rank == 0 and world == 1:
        if not args.no_batched:
            batched = {"u32": batched_bench(mgs, torch, ctx, "u32"),
                       "f32": batched_bench(mgs, torch, ctx, "f32", with_plain=False)}
        if not args.no_served:
            served = served_bench(mgs, torch)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        orc = load_oracle()
        if orc.ref_available():
            v, threads, times = cpu_reference_sort(orc, keys_np, budget_s=12.0, max_reps=3)
            cpu = {"value": v, "unit": "keys/s", "cores": threads, "kind": "reference",
                   "sample": f"the whole workload ({n} keys), {len(times)} runs, median "
                             f"(reference gnu_parallel sort, src/sort_benchmark.cu:103-108)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "keys/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": sort_ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "u32", "data": "synthetic (reference DataGenerator, seeded)",
            "config": {"workload": WORKLOAD, "keys_per_gpu": n, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (4 GiB per step)",
                       "timing": "CUDA events around each sort on its stream; input restored from a pristine "
                                 "device copy before each step, outside the timed region",
                       "sort_hbm_alg_gbs": sort_alg_bytes / (sort_ms / 1e3) / 1e9,
                       "sort_roofline_frac": sort_alg_bytes / (sort_ms / 1e3) / 1e9 / peak,
                       "verified": ok and e2e_ok},
            "roofline": roof,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "keys/s", "h2d_bytes_per_step": 4 * n, "d2h_bytes_per_step": 4 * n,
                    "api": "mgs_sort_host (TanasicSort, one GPU)", "steps": len(e2e_times)},
            "batched": batched,
            "served": served,
            "gpu_launches": launches,
            "kernel_ms": {k: {"launches": v[0], "total_ms": v[1]} for k, v in ktimes.items()},
            "clocks": clocks.summary(),
        }
        print(json.dumps(line))

    del work, pristine, temp
    ctx.close()
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
