"""The N-process path of bench.py on CPU: two gloo ranks agree on the slowest
rank's time (all-reduce MAX) and on the whole-job throughput, and the reference
arm does its work on rank 0 only (the other ranks exit without output)."""
import importlib.util
import multiprocessing as mp
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def load_bench():
    spec = importlib.util.spec_from_file_location("bench_module", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world)
    try:
        bench = load_bench()
        dist.barrier()
        slowest = bench.max_over_ranks(dist, world, 100.0 + 7.5 * rank, "cpu")
        out.put((rank, slowest, bench.job_keys_per_s(world, 1 << 30, 5, slowest / 1e3)))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_gloo_ranks_take_the_slowest_time():
    ctx = mp.get_context("spawn")
    out = ctx.Queue()
    port = free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(out.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [107.5, 107.5]
    assert all(abs(g[2] - 2 * (1 << 30) * 5 / 0.1075) < 1 for g in got)


def test_single_rank_needs_no_process_group():
    bench = load_bench()
    assert bench.max_over_ranks(None, 1, 42.0, "cpu") == 42.0
    assert bench.job_keys_per_s(1, 1000, 4, 2.0) == 2000.0


def test_reference_arm_runs_on_rank_zero_only():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2",
                        "--steps", "1", "--warmup", "0"], env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
