"""GPU bar of the reference's own sort path: thrust::sort -> CUB DeviceRadixSort
(src/tanasic_sort.cuh:264-266), compiled from the reference sources into
oracle/_ref by oracle/Makefile, timed with CUDA events on a device-resident
array. Test infrastructure: it measures the reference, never the engine.

python oracle/cub_bar.py [--log2n 30] [--reps 5]

Prints one JSON line: CUB milliseconds per sort of 2^log2n uint32 keys and of
2^(log2n-1) uint64 keys (the reference DataGenerator inputs of the engine's
benchmark), and whether the results are sorted.
"""
import argparse
import importlib.util
import json
import os
import statistics
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--log2n", type=int, default=30)
    ap.add_argument("--reps", type=int, default=5)
    args = ap.parse_args()
    import torch
    sys.path.insert(0, HERE)
    import oracle
    if not oracle.ref_available():
        print(json.dumps({"unavailable": "oracle/_ref not built"}))
        return
    spec = importlib.util.spec_from_file_location("mgs", os.path.join(ROOT, "multi-gpu-sorting_b200", "mgs.py"))
    mgs = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mgs)
    out = {}
    for dtype, code, storage, n in (("u32", 0, np.int32, 1 << args.log2n), ("u64", 3, np.int64, 1 << (args.log2n - 1))):
        keys = mgs.generate(dtype, "uniform" if dtype == "u32" else "full-uniform", 2147483647, n)
        src = torch.from_numpy(keys.view(storage)).cuda()
        work = torch.empty_like(src)
        _, need = oracle.ref_cub_sort_device_ms(code, src.data_ptr(), work.data_ptr(), n)
        temp = torch.empty(need, dtype=torch.uint8, device="cuda")
        times = []
        for i in range(args.reps + 1):
            torch.cuda.synchronize()
            ms, _ = oracle.ref_cub_sort_device_ms(code, src.data_ptr(), work.data_ptr(), n, temp.data_ptr(), need)
            if i > 0:
                times.append(ms)
        k = work.to(torch.int64) & 0xFFFFFFFF if dtype == "u32" else work ^ (-(1 << 63))
        out[f"cub_{dtype}_2^{n.bit_length() - 1}_ms"] = statistics.median(times)
        out[f"cub_{dtype}_sorted"] = bool((k[1:] >= k[:-1]).all())
        del src, work, temp, k
    print(json.dumps(out))


if __name__ == "__main__":
    main()
