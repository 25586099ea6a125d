"""Counting-wave microbenchmark: one wave of b single-item nodes against d items over a
random bitmap of N transactions, with each counter forced; prints the time and rate of
each counter and checks that all counters return identical counts.

    python -m tensorfim_b200.countbench [--nodes 512] [--items 1024] [--bits 262144]
                                        [--density 0.5] [--counters i8,tensor,lop3] [--reps 3]

Rate unit: bit-ops/s = b x d x N / time (the reference microbench's unit,
code/microbench/bmma_bench.cu:400).  Times are CUDA events around tfim_count_wave_device
(mask build + counting + threshold count), median of --reps after one warm-up.
"""
from __future__ import annotations

import argparse
import json
import statistics

import numpy as np

from .engine import Database


def run(nodes: int, items: int, bits: int, density: float = 0.5, counters=("i8", "tensor", "lop3"), reps: int = 3,
        seed: int = 7) -> dict:
    import torch
    rng = np.random.Generator(np.random.PCG64(seed))
    words = (bits + 31) // 32
    rows = rng.integers(0, 2 ** 32, size=(items, words), dtype=np.uint64).astype(np.uint32)
    if density < 0.5:   # AND of two random words: 25%
        rows &= rng.integers(0, 2 ** 32, size=(items, words), dtype=np.uint64).astype(np.uint32)
    out = {"nodes": nodes, "items": items, "bits": bits, "counters": {}}
    ref = None
    with Database.from_bitmap(rows, bits, items) as db:
        lists = torch.arange(nodes, dtype=torch.int32, device="cuda") % items
        offs = torch.arange(nodes + 1, dtype=torch.int64, device="cuda")
        for counter in counters:
            counts = torch.zeros((nodes, items), dtype=torch.int32, device="cuda")
            nfreq = torch.zeros(nodes, dtype=torch.int32, device="cuda")
            db.set_counter(counter)
            ts = []
            for k in range(reps + 1):
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                db.count_wave_device(lists.data_ptr(), offs.data_ptr(), nodes, 1, 1, counts.data_ptr(), nfreq.data_ptr())
                e1.record()
                torch.cuda.synchronize()
                if k:
                    ts.append(e0.elapsed_time(e1) / 1000.0)
            c = counts.cpu().numpy()
            if ref is None:
                ref = c
            assert (c == ref).all(), f"{counter} counts differ"
            t = statistics.median(ts)
            out["counters"][counter] = {"seconds": t, "bitops_per_s": nodes * items * bits / t}
    return out


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--nodes", type=int, default=512)
    ap.add_argument("--items", type=int, default=1024)
    ap.add_argument("--bits", type=int, default=1 << 18)
    ap.add_argument("--density", type=float, default=0.5)
    ap.add_argument("--counters", default="i8,tensor,lop3")
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    print(json.dumps(run(a.nodes, a.items, a.bits, a.density, a.counters.split(","), a.reps)))


if __name__ == "__main__":
    main()
