"""Generates tests/golden/generator.json from the reference's own DataGenerator.

Run in a checkout where oracle/_ref/libref.so was built from the reference's
sources (make -C oracle): python tests/golden/make_golden.py

Each entry is the SHA-256 of DataGenerator(seed).ComputeDistribution<T>(n,
distribution) (src/data_generator.cuh:18-36) as produced by the reference. For
"nearly-sorted" the reference reads each block's successor element while the
next OpenMP thread may already have raised it (a data race at the 127 block
boundaries, src/data_generator.cuh:140-159), so the hash is taken after zeroing
the last element of every generator block.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(HERE, "..", "..", "oracle"))
import oracle  # noqa: E402

DTYPES = ["uint32", "int32", "float32", "uint64", "int64", "float64"]
DISTS = ["uniform", "normal", "zero", "staggered", "sorted", "reverse-sorted", "nearly-sorted", "bucket-sorted"]
SIZES = [10, 129, 1000, 65537]
SEEDS = [2147483647, 7]


def race_positions(n: int, threads: int = 128):
    """Last index of each schedule(static) block of the n-1 nearly-sorted iterations."""
    m = n - 1
    q, r = divmod(m, threads)
    out = []
    for t in range(threads):
        b = t * (q + 1) if t < r else t * q + r
        e = b + (q + 1 if t < r else q)
        if e > b:
            out.append(e - 1)
    return np.array(out, dtype=np.int64)


def digest(a: np.ndarray, dist: str) -> str:
    a = a.copy()
    if dist == "nearly-sorted" and a.size > 1:
        a[race_positions(a.size)] = 0
    return hashlib.sha256(a.tobytes()).hexdigest()


def main():
    entries = []
    for dt in DTYPES:
        for dist in DISTS:
            for n in SIZES:
                for seed in SEEDS:
                    a = oracle.ref_generate(np.dtype(dt), dist, seed, n)
                    entries.append({"dtype": dt, "distribution": dist, "n": n, "seed": seed,
                                    "sha256": digest(a, dist)})
    with open(os.path.join(HERE, "generator.json"), "w") as f:
        json.dump({"source": "reference DataGenerator (src/data_generator.cuh) via oracle/_ref",
                   "entries": entries}, f, indent=0)
    print(f"wrote {len(entries)} entries")


if __name__ == "__main__":
    main()
