#!/usr/bin/env python
"""Benchmark of the MFI mining hot path on B200.

Workload (default): the sparse long-tail configuration -- 1,000,000 transactions over
40,000 items, minimum support 0.05% (seeded synthetic data, tensorfim_b200.synth cfg 4).
It is the largest of the five benchmark configurations by counting work; the dense 70k
configuration is a 9-node search and the replicated 12.5M configuration has no frequent
item at 85% (its largest item support is 0.711), so neither exercises the counters.

One step = one complete mine of the database (search + every support count), bitmap
already resident in HBM.  `value` is throughput in reference-equivalent supports per
second: the number of supports the reference engine counts for this database (its nodes
x survivors, measured by the plain engine, which runs the reference's search) divided by
the resident batched engine's mine time with the learned lookahead proposal, summed over
ranks (each rank mines its own copy: weak scaling).  `e2e` is the same metric through the C ABI from pinned host buffers: build
the device database from the host CSR, mine, read the MFIs back, every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tfim|reference] [--workload cfg4]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}

WORKLOADS = {
    "cfg4": dict(cfg=4, kw={}, minsup=0.0005,
                 desc="sparse long-tail DB: 1,000,000 tx x 40,000 items, Poisson(10)+1 lengths, 2,000 patterns, minsup 0.05%"),
    "cfg5": dict(cfg=5, kw={}, minsup=0.70,
                 desc="dense categorical DB: 2,000,000 tx x 60 groups (~500 items), minsup 70%"),
    "cfg1": dict(cfg=1, kw={}, minsup=0.10, desc="dense categorical DB: 10,000 tx x 23 groups x 5 values, minsup 10%"),
    "cfg2": dict(cfg=2, kw={}, minsup=0.90, desc="dense categorical DB: 70,000 tx x 43 groups x 3 values, minsup 90%"),
    "cfg3": dict(cfg=3, kw={}, minsup=0.85,
                 desc="replicated dense DB: 49,000 x 256 = 12,544,000 tx, 74 Zipf(1.3) groups, minsup 85%"),
}


def peaks() -> tuple[dict, str]:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return dict(PEAKS_FALLBACK), "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("timestamp,index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.3)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.f.read().splitlines():
            parts = [x.strip() for x in ln.split(",")]
            if len(parts) < 10:
                continue
            try:
                sm.append(float(parts[2]))
                mx.append(float(parts[3]))
            except ValueError:
                continue
            for k, name in enumerate(names):
                if parts[6 + k].lower() == "active":
                    reasons.add(name)
        self.f.close()
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def load_traffic(kernel: str):
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(kernel)
    return None


def make_db(name: str):
    from tensorfim_b200 import synth
    w = WORKLOADS[name]
    return synth.generate(w["cfg"], **w["kw"]), w


# ------------------------------------------------------------------------------ reference arm
def run_reference_arm(args, rank: int, world: int) -> int:
    """The reference's own CPU implementation (oracle/_ref/tfim_ref_mt: code/engine/src/
    kernel_bitmap.cu compiled unmodified, RUN_MODE 2 with every node on its multithreaded
    CPU counter), on a bounded sample of the workload: the same generator at --ref-scale of
    the rows (default 2%) and the same minimum support.  Under torchrun only rank 0 runs it;
    the other ranks exit 0 without work.  Its per-support cost is linear in the transaction count,
    so supports are scaled by N_sample/N_full to full-workload supports."""
    if rank != 0:
        return 0
    from oracle import oracle
    from tensorfim_b200 import synth
    w = WORKLOADS[args.workload]
    if not os.path.exists(oracle.REF_MT):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/tfim_ref_mt was not built (reference tree absent at build time)"}))
        return 0
    scale = args.ref_scale
    sample = synth.generate(w["cfg"], **dict(w["kw"], scale=scale)) if w["cfg"] != 3 else synth.generate(3, replicas=max(1, int(256 * scale)))
    full_rows = {1: 10_000, 2: 70_000, 3: 12_544_000, 4: 1_000_000, 5: 2_000_000}[w["cfg"]]
    threads = os.cpu_count() or 1
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "sample.txt")
        synth.write_fimi(path, sample)
        odb = oracle.OracleDB(path, w["minsup"])
        odb.mine(threads)
        nodes = odb.nodes
        d_surv = odb.info()["n_survivors"]
        n_red = odb.info()["trans_num_reduced"]
        odb.close()
        supports_full_eq = nodes * d_surv * (sample.n_rows / full_rows)
        times = []
        for k in range(args.warmup + args.steps):
            _, hdr = oracle.run_reference(path, w["minsup"], binary=oracle.REF_MT, threads=threads, timeout=1800)
            if k >= args.warmup:
                times.append(float(hdr["computation_time(s)"]))
    t = statistics.mean(times)
    v = supports_full_eq / t
    unit = "supports/s"
    out = {
        "impl": "reference", "metric": "MFI mine time (s) & supports/s, batched+learned vs plain on 1 B200, set-identical",
        "value": v, "unit": unit, "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": t * 1000, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic", "config": {"workload": args.workload, "desc": w["desc"], "minsup": w["minsup"]},
        "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": "reference",
                         "sample": f"reference multithreaded CPU engine on the same generator at {scale:.0%} of the rows "
                                   f"({sample.n_rows} tx, {n_red} reduced, {d_surv} survivors, {nodes} nodes); supports scaled "
                                   f"by {sample.n_rows}/{full_rows} to full-size per-support cost; computation_time(s) from its results file"},
        "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))
    return 0


# ------------------------------------------------------------------------------ our arm
def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tfim", choices=["tfim", "reference"])
    ap.add_argument("--workload", default="cfg4", choices=sorted(WORKLOADS))
    ap.add_argument("--counter", default="auto", choices=["auto", "lop3", "tensor", "proj"])
    ap.add_argument("--engine", default="resident", choices=["batched", "resident"])
    ap.add_argument("--lookahead", default="learned", choices=["off", "filtered", "learned", "all"])
    ap.add_argument("--ref-scale", type=float, default=0.02)
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":
        return run_reference_arm(args, rank, world)

    import torch
    import torch.distributed as dist
    import tensorfim_b200 as tf
    from tensorfim_b200 import replicas

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, device="cuda")

    db0, w = make_db(args.workload)
    # pinned host copies of the inputs (the e2e path copies them every step)
    h_off = torch.from_numpy(db0.offsets).pin_memory()
    h_items = torch.from_numpy(db0.items).pin_memory()
    off_np, items_np = h_off.numpy(), h_items.numpy()
    h2d_bytes = off_np.nbytes + items_np.nbytes
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")   # > 126 MB L2

    db = tf.Database.from_csr(off_np, items_np, w["minsup"], device=local)
    info = db.info
    mine_kw = dict(engine=args.engine, counter=args.counter, lookahead=args.lookahead)
    for _ in range(args.warmup):
        db.mine(**mine_kw)
    barrier()
    clocks = Clocks(local) if rank == 0 else None
    step_ms, kern_ms, stats = [], [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        r = db.mine(**mine_kw)
        step_ms.append(r.stats["device_ms"])
        kern_ms.append(r.stats["kernel_ms"])
        stats.append(r.stats)
    barrier()
    clk = clocks.stop() if clocks else None
    batched = r
    ms = max_over_ranks(statistics.mean(step_ms))

    # the plain engine (the reference's search, one counted node per launch): defines the
    # reference-equivalent supports of this database and the batched-vs-plain speedup
    plain = None
    if not args.no_plain:
        plain = db.mine(engine="plain")
        ref_supports = plain.stats["supports"]
        identical = plain.as_dict() == batched.as_dict()
    else:
        ref_supports = batched.stats["supports"]
        identical = None
    value = replicas.job_throughput(ref_supports, ms, world)

    # end to end through the C ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        e2e_ms = []
        d2h = 0
        for k in range(max(1, args.warmup) + args.steps):
            flush.zero_()
            barrier()
            t0 = time.perf_counter()
            d = tf.Database.from_csr(off_np, items_np, w["minsup"], device=local)
            res = d.mine(**mine_kw)
            d.close()
            t1 = time.perf_counter()
            if k >= max(1, args.warmup):
                e2e_ms.append((t1 - t0) * 1000.0)
            d2h = res.items.nbytes + res.offsets.nbytes + res.supports.nbytes
        e2e_t = max_over_ranks(statistics.mean(e2e_ms))
        e2e = {"value": replicas.job_throughput(ref_supports, e2e_t, world), "unit": "supports/s", "h2d_bytes_per_step": int(h2d_bytes),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_t,
               "timing": "host wall clock around open (H2D + device ingest) + mine + MFI read-back + close"}

    # roofline of the counting kernels over the timed steps
    pk, pk_src = peaks()
    tot_bytes = sum(s["bytes_alg"] for s in stats)
    tot_bitops = sum(s["bit_ops"] for s in stats)
    tot_kms = sum(kern_ms)
    tot_launch = sum(s["count_launches"] for s in stats)
    achieved = tot_bytes / (tot_kms / 1000.0) / 1e9 if tot_kms > 0 else 0.0
    traffic = load_traffic("count")
    roofline = {"bound": "hbm", "achieved": achieved, "peak": pk["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / pk["hbm_gbs"], "peak_source": pk_src,
                "traffic": traffic, "bytes_alg_per_launch": tot_bytes / max(1, tot_launch),
                "kernel_ms_per_launch": tot_kms / max(1, tot_launch),
                "bitops_per_s": tot_bitops / (tot_kms / 1000.0) if tot_kms > 0 else 0.0,
                "kernel": "counting launches of the search (k_count_lop3 / k_count_b1 / k_pair_count)"}

    # CPU baseline: the oracle port (multithreaded AND+popcount, the reference's search)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        from oracle import oracle
        threads = os.cpu_count() or 1
        odb = oracle.OracleDB(None, w["minsup"], csr=(off_np, items_np))
        nodes, secs = odb.mine_sample(args.cpu_budget, threads)
        d_surv = odb.info()["n_survivors"]
        odb.close()
        cpu = {"value": nodes * d_surv / secs, "unit": "supports/s", "cores": threads, "kind": "port",
               "sample": f"oracle restatement (tfim_oracle.c, OpenMP) on the full database, root subtrees in the reference's "
                         f"pop order for a {args.cpu_budget:.0f} s budget: {nodes} nodes x {d_surv} survivors in {secs:.1f} s"}

    gpu_launches = sum(s["launches"] for s in stats)
    out = {
        "metric": "MFI mine time (s) & supports/s, batched+learned vs plain on 1 B200, set-identical",
        "value": value, "unit": "supports/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "minsup": w["minsup"], "rows": db0.n_rows,
                   "reduced_rows": info["trans_num_reduced"], "survivors": info["n_survivors"],
                   "bitmap_bytes": int(info["n_dense"]) * int(info["words_per_row"]) * 4,
                   "l2": "inputs larger than L2 (bitmap) and a 256 MB L2 flush before every timed step",
                   "engine": args.engine, "counter": args.counter, "lookahead": args.lookahead,
                   "parallelism": f"{world} independent database replicas, one per GPU"},
        "mine_time_s": ms / 1000.0,
        "plain_mine_time_s": plain.stats["device_ms"] / 1000.0 if plain else None,
        "speedup_vs_plain": (plain.stats["device_ms"] / ms) if plain else None,
        "set_identical_to_plain": identical,
        "n_mfi": len(batched),
        "reference_supports_per_db": ref_supports,
        "counted_supports_per_db": batched.stats["supports"],
        "stats": {k: v for k, v in batched.stats.items()},
        "plain_stats": plain.stats if plain else None,
        "roofline": roofline,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "clocks": clk,
    }
    db.close()
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
