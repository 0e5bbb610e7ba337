"""The sort_benchmark CLI keeps the reference's options, validation and CSV line
(src/sort_benchmark.cu:130-228, src/argument_limits.cuh)."""
import csv
import io
import os
import subprocess

import pytest

from conftest import PKG

CLI = os.path.join(PKG, "bin", "sort_benchmark")
COLUMNS = ["num_elements", "algorithm", "gpus", "data_type", "distribution_type", "distribution_seed", "num_threads",
           "chunk_size", "merge_group_size", "num_buffers", "memory_allocation", "sort_phase", "memory_deallocation",
           "total"]


def run(*args):
    return subprocess.run([CLI, *map(str, args)], capture_output=True, text=True, timeout=600)


def parse(line):
    row = next(csv.reader(io.StringIO(line)))
    assert len(row) == len(COLUMNS), row
    return dict(zip(COLUMNS, row))


@pytest.mark.parametrize("algorithm", ["gnu_parallel", "std"])
@pytest.mark.parametrize("data_type", ["int", "long", "float", "double", "uint32", "uint64"])
def test_cpu_algorithms_print_one_csv_line(algorithm, data_type):
    r = run(20000, "--algorithm", algorithm, "--data_type", data_type, "--distribution_type", "normal",
            "--num_threads", 2)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 1, r.stdout  # no "Error: Invalid sort order."
    row = parse(lines[0])
    assert row["num_elements"] == "20000" and row["algorithm"] == algorithm and row["gpus"] == "0"
    assert row["data_type"] == data_type and row["distribution_seed"] == "2147483647"
    assert float(row["total"]) >= float(row["sort_phase"]) > 0


@pytest.mark.parametrize("args,needle", [
    (["abc"], "Invalid <num_elements>"),
    (["10", "--algorithm", "quicksort"], "Invalid <algorithm>"),
    (["10", "--gpus", "0,1,2"], "Invalid <gpus>"),
    (["10", "--gpus", "{0,0}"], "Invalid <gpus>"),
    (["10", "--data_type", "short"], "Invalid <data_type>"),
    (["10", "--distribution_type", "poisson"], "Invalid <distribution_type>"),
    (["10", "--num_buffers", "4"], "Invalid <num_buffers>"),
    (["10", "--chunks", "3"], "Invalid <chunks>"),
])
def test_invalid_arguments_print_usage(args, needle):
    r = run(*args)
    assert r.returncode == 1
    assert needle in r.stdout and "Usage:" in r.stdout


def test_help_and_unavailable_baselines():
    assert run("--help").returncode == 1
    r = run(10, "--algorithm", "paradis")
    assert r.returncode == 1 and "not available" in r.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("args", [
    ["--algorithm", "tanasic"],
    ["--algorithm", "tanasic", "--chunks", "8", "--data_type", "float"],
    ["--algorithm", "thrust", "--data_type", "uint64", "--distribution_type", "zipf"],
    ["--algorithm", "gowanlock", "--chunk_size", "100000", "--num_buffers", "3"],
    ["--algorithm", "gowanlock", "--chunk_size", "250000", "--data_type", "double"],
])
def test_engine_algorithms_sort(args):
    r = run(1_000_003, *args)
    assert r.returncode == 0, r.stdout + r.stderr
    lines = r.stdout.strip().splitlines()
    assert len(lines) == 1, r.stdout
    row = parse(lines[0])
    assert float(row["sort_phase"]) > 0
