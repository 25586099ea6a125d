#!/usr/bin/env python
"""Benchmark of the MFI mining hot path on B200.

Workload (default, `cfg3dev`): the replicated dense configuration at full size -- 49,000
base rows x 256 exact replicas = 12,544,000 transactions, 74 Zipf(1.3) attribute groups of
2-60 values (~2,100 item ids) -- with the minimum support lowered from 85% to 6% (a labelled
deviation: at 85% no item is frequent).  271 frequent items, a 1.57 MB bitmap row per item,
40,760 nodes of the reference's search, 31,589 MFIs.  `--workload cfg4` runs the sparse
1,000,000 x 40,000 configuration.  Seeded synthetic data of the configurations' shapes
(tensorfim_b200.synth) stand in for the reference's FIMI files.

One step = one complete mine of the database (search + every support count), the bitmap
resident in HBM; a 256 MB L2 flush precedes every timed step and the bitmap itself is
larger than L2.  `value` is reference-equivalent supports per second: the supports the
reference's search counts on this database (its nodes x survivors, counted by the plain
engine, which runs that search) over the batched engine's mine time with the learned
lookahead proposal, summed over ranks (each rank mines its own copy: weak scaling).  The
supports the batched engine actually counts per second are reported beside it.  `e2e` is
the same metric through the C ABI from pinned host buffers: build the device database from
the host CSR, mine, read the MFIs back, close, every step.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl tfim|reference] [--workload cfg3dev]
"""
from __future__ import annotations

import argparse
import gzip
import json
import os
import statistics
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from tensorfim_b200 import measure, synth  # noqa: E402

METRIC = "MFI mine time (s) & supports/s, batched+learned vs plain on 1 B200, set-identical"

# ref_supports: supports the reference's search counts on the database (its node count x
# the survivors), as the plain engine counts them (checked at every run)
WORKLOADS = {
    "cfg3dev": dict(cfg=3, kw={}, minsup=synth.CFG3_DEVIATION_MINSUP, ref_supports=40_760 * 271,
                    golden="cfg3_base_t06", golden_factor=256,
                    desc="replicated dense DB at full size: 49,000 x 256 = 12,544,000 tx, 74 Zipf(1.3) groups "
                         "(~2,100 items); minsup lowered from 85% (no frequent item) to 6%: labelled deviation"),
    "cfg4": dict(cfg=4, kw={}, minsup=0.0005, ref_supports=14_072 * 6_162,
                 desc="sparse long-tail DB: 1,000,000 tx x 40,000 items, Poisson(10)+1 lengths, 2,000 patterns, "
                      "minsup 0.05%"),
    "cfg5": dict(cfg=5, kw={}, minsup=0.70, ref_supports=150 * 38,
                 desc="dense categorical DB: 2,000,000 tx x 60 groups (~500 items), minsup 70%"),
    "cfg1": dict(cfg=1, kw={}, minsup=0.10, ref_supports=3_164 * 69, golden="cfg1_full",
                 desc="dense categorical DB: 10,000 tx x 23 groups x 5 values, minsup 10%"),
    "cfg2": dict(cfg=2, kw={}, minsup=0.90, ref_supports=9 * 9, golden="cfg2_full",
                 desc="dense categorical DB: 70,000 tx x 43 groups x 3 values, minsup 90%"),
    "cfg3": dict(cfg=3, kw={}, minsup=0.85, ref_supports=None,
                 desc="replicated dense DB: 49,000 x 256 = 12,544,000 tx, 74 Zipf(1.3) groups, minsup 85% "
                      "(no frequent item)"),
}
DEFAULT_WORKLOAD = "cfg3dev"


def make_db(name: str):
    w = WORKLOADS[name]
    return synth.generate(w["cfg"], **w["kw"]), w


def golden_mfis(w) -> dict | None:
    """The reference's MFIs for the workload (a fixture the reference produced at base size),
    supports scaled to the replicated database."""
    if not w.get("golden"):
        return None
    p = os.path.join(ROOT, "tests", "golden", w["golden"] + ".json.gz")
    if not os.path.exists(p):
        return None
    with gzip.open(p, "rt") as f:
        fx = json.load(f)
    k = w.get("golden_factor", 1)
    return {frozenset(s): f * k for s, f in fx["mfis"]}


def write_workload_text(path: str, name: str) -> None:
    w = WORKLOADS[name]
    if name in ("cfg3dev", "cfg3"):
        synth.write_fimi_replicated(path, synth.cfg3_base(), 256)
    else:
        synth.write_fimi(path, synth.generate(w["cfg"], **w["kw"]))


# ------------------------------------------------------------------------------ reference arm
def _phase_line(text: str) -> dict | None:
    for ln in text.splitlines():
        if ln.startswith("BMMA phase ms:"):
            out = {}
            for tok in ln.split(":", 1)[1].split():
                k, _, v = tok.partition("=")
                try:
                    out[k] = float(v)
                except ValueError:
                    pass
            return out
    return None


def run_reference_arm(args, rank: int, world: int) -> int:
    """The reference's own CPU implementation (oracle/_ref/tfim_ref_mt: code/engine/src/
    kernel_bitmap.cu compiled unmodified, RUN_MODE 2 with every node on its multithreaded CPU
    counter, all host threads) mines the full workload file; a step is one run of it, and runs
    stop once --ref-budget seconds are spent (at least one; `steps` reports the runs made).
    Beside it, the reference's GPU engines rebuilt for sm_100a (the BMMA wave engine,
    kernel_bmma.cu, and the per-node GPU engine, kernel_bitmap.cu RUN_MODE 1) mine the same
    file once each on this GPU.  Under torchrun only rank 0 runs; the other ranks exit 0."""
    if rank != 0:
        return 0
    from oracle import oracle
    w = WORKLOADS[args.workload]
    if not os.path.exists(oracle.REF_MT):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/tfim_ref_mt was not built (reference tree absent at build time)"}))
        return 0
    threads = os.cpu_count() or 1
    gold = golden_mfis(w)
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, args.workload + ".txt")
        write_workload_text(path, args.workload)
        comp, total, runs = [], [], 0
        t_start = time.perf_counter()
        ident_cpu = None
        n_mfi = None
        while runs < max(1, args.warmup + args.steps):
            so = {}
            mfis, hdr = oracle.run_reference(path, w["minsup"], binary=oracle.REF_MT, threads=threads,
                                             timeout=3600, in_place=True, stdout=so)
            comp.append(float(hdr["computation_time(s)"]))
            total.append(so["wall_s"])
            n_mfi = len(mfis)
            if gold is not None:
                ident_cpu = mfis == gold
            runs += 1
            if time.perf_counter() - t_start > args.ref_budget:
                break
        gpu = {}
        if not args.no_ref_gpu:
            for name, binary in (("bmma", oracle.REF_BMMA), ("pernode", oracle.REF_GPU)):
                if not os.path.exists(binary):
                    gpu[name] = {"unavailable": f"{os.path.basename(binary)} was not built"}
                    continue
                so = {}
                try:
                    mfis, hdr = oracle.run_reference(path, w["minsup"], binary=binary, timeout=1800, in_place=True,
                                                     stdout=so)
                    gpu[name] = {"computation_s": float(hdr["computation_time(s)"]),
                                 "preprocessing_s": float(hdr["preprocessing_time(s)"]),
                                 "total_s": float(hdr["total_time(s)"]), "wall_s": so["wall_s"],
                                 "n_mfi": len(mfis), "set_identical_to_reference_fixture":
                                     (mfis == gold) if gold is not None else None,
                                 "phase_ms": _phase_line(so["text"])}
                except Exception as e:   # a failed comparator is reported, not fatal
                    gpu[name] = {"error": repr(e)[:300]}
    t = statistics.mean(comp)
    ref_sup = w["ref_supports"]
    v = ref_sup / t if ref_sup else None
    unit = "supports/s"
    out = {
        "impl": "reference", "metric": METRIC,
        "value": v, "unit": unit, "n_gpus": world, "steps": runs, "warmup": 0,
        "steps_requested": args.steps, "warmup_requested": args.warmup,
        "ms_per_step": t * 1000, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "minsup": w["minsup"], "same_config": True},
        "mine_time_s": t, "wall_s_per_run": statistics.mean(total), "n_mfi": n_mfi,
        "set_identical_to_reference_fixture": ident_cpu,
        "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": "reference",
                         "sample": f"the reference's multithreaded CPU engine (kernel_bitmap.cu RUN_MODE 2, every node on "
                                   f"the CPU counter) on the full {args.workload} file, {runs} run(s) within a "
                                   f"{args.ref_budget:.0f} s budget; computation_time(s) from its results file"},
        "e2e": {"value": (ref_sup / statistics.mean(total)) if ref_sup else None, "unit": unit,
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                "timing": "wall clock of the reference process: parse, preprocessing, mining, results file"},
        "reference_gpu": gpu,
    }
    print(json.dumps(out))
    return 0


# ------------------------------------------------------------------------------ our arm
def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="tfim", choices=["tfim", "reference"])
    ap.add_argument("--workload", default=DEFAULT_WORKLOAD, choices=sorted(WORKLOADS))
    ap.add_argument("--counter", default="auto", choices=["auto", "lop3", "tensor", "proj", "i8"])
    ap.add_argument("--engine", default="resident", choices=["batched", "resident"])
    ap.add_argument("--lookahead", default="learned", choices=["off", "filtered", "learned", "all"])
    ap.add_argument("--graphs", type=int, default=0)
    ap.add_argument("--plain-runs", type=int, default=2)
    ap.add_argument("--ref-budget", type=float, default=240.0)
    ap.add_argument("--no-ref-gpu", action="store_true")
    ap.add_argument("--cpu-budget", type=float, default=15.0)
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-ablation", action="store_true")
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
    dev = torch.device("cuda", local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    def max_over_ranks(x: float) -> float:
        return replicas.max_over_ranks(x, device="cuda")

    pk, pk_src = measure.peaks()
    i8_macs = measure.i8_gemm_peak(dev)
    i8_src = "measured (torch._int_mm 8192^3 on this GPU, best of 10)" if i8_macs else None
    sm_count = torch.cuda.get_device_properties(dev).multi_processor_count

    db0, w = make_db(args.workload)
    # pinned host copies of the inputs (the e2e path copies them every step)
    h_off = torch.from_numpy(db0.offsets).pin_memory()
    h_items = torch.from_numpy(db0.items).pin_memory()
    off_np, items_np = h_off.numpy(), h_items.numpy()
    h2d_bytes = off_np.nbytes + items_np.nbytes
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)   # > 126 MB L2

    db = tf.Database.from_csr(off_np, items_np, w["minsup"], device=local)
    info = db.info
    mine_kw = dict(engine=args.engine, counter=args.counter, lookahead=args.lookahead, graphs=bool(args.graphs))
    for _ in range(max(3, args.warmup)):
        db.mine(**mine_kw)
    barrier()
    clocks = measure.Clocks(local) if rank == 0 else None
    step_ms, stats = [], []
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        r = db.mine(**mine_kw)
        step_ms.append(r.stats["device_ms"])
        stats.append(r.stats)
    barrier()
    clk = clocks.stop() if clocks else None
    batched = r
    ms = max_over_ranks(statistics.mean(step_ms))

    # the plain engine (the reference's search, one counted node per launch): the reference's
    # support count for this database and the batched-vs-plain ratio
    plain, plain_ms = None, None
    if not args.no_plain:
        pm = []
        for _ in range(max(1, args.plain_runs)):
            flush.zero_()
            torch.cuda.synchronize()
            plain = db.mine(engine="plain")
            pm.append(plain.stats["device_ms"])
        plain_ms = statistics.mean(pm)
        ref_supports = plain.stats["supports"]
        identical = plain.as_dict() == batched.as_dict()
    else:
        ref_supports = w["ref_supports"] or batched.stats["supports"]
        identical = None
    gold = golden_mfis(w)
    ident_gold = (batched.as_dict() == gold) if gold is not None else None
    value = replicas.job_throughput(ref_supports, ms, world)
    counted = statistics.mean(s["supports"] for s in stats)

    # the lookahead ablation: learned proposal, tail-pair filter, none; and the graph loop
    ablation = None
    if not args.no_ablation and rank == 0:
        ablation = {}
        for name, kw in (("learned", dict(lookahead="learned")), ("filtered", dict(lookahead="filtered")),
                         ("off", dict(lookahead="off")), ("learned_graph", dict(lookahead="learned", graphs=True))):
            t, last = [], None
            for _ in range(3):
                flush.zero_()
                torch.cuda.synchronize()
                last = db.mine(engine=args.engine, counter=args.counter, **kw)
                t.append(last.stats["device_ms"])
            ablation[name] = {"mine_ms": statistics.median(t), "counted_supports": last.stats["supports"],
                              "nodes": last.stats["nodes"], "lookaheads": last.stats["lookaheads"],
                              "lookahead_hits": last.stats["lookahead_hits"], "waves": last.stats["waves"],
                              "identical": last.as_dict() == batched.as_dict()}

    # the benchmark database is closed before the end-to-end steps, as a caller opening
    # databases in sequence would: with both open, two sets of search pools (tens of GB on
    # this workload) exceed the device pool's cache and every step remaps memory
    db.close()

    # end to end through the C ABI from pinned host memory
    e2e = None
    if not args.no_e2e:
        e2e_ms, ph = [], {"open_ms": [], "mine_ms": [], "close_ms": []}
        first_paths = []
        d2h = 0
        n_e2e = max(3, args.steps)
        for k in range(max(1, args.warmup) + n_e2e):
            flush.zero_()
            barrier()
            t0 = time.perf_counter()
            d = tf.Database.from_csr(off_np, items_np, w["minsup"], device=local)
            t1 = time.perf_counter()
            res = d.mine(**mine_kw)
            t2 = time.perf_counter()
            d.close()
            t3 = time.perf_counter()
            if k >= max(1, args.warmup):
                e2e_ms.append((t3 - t0) * 1000.0)
                ph["open_ms"].append((t1 - t0) * 1000.0)
                ph["mine_ms"].append((t2 - t1) * 1000.0)
                ph["close_ms"].append((t3 - t2) * 1000.0)
                ph.setdefault("mine_device_ms", []).append(res.stats["device_ms"])
                ph.setdefault("mine_readback_ms", []).append(res.stats["readback_ms"])
                ph.setdefault("mine_setup_ms", []).append(res.stats["setup_ms"])
                # where the first mine on a freshly opened database spends its time
                for key in ("kernel_ms", "host_ms", "sync_ms", "top_ms", "pack_ms", "expand_ms", "mask_ms"):
                    ph.setdefault("mine_" + key, []).append(res.stats[key])
                first_paths.append(res.stats["path_ms"])
            d2h = res.items.nbytes + res.offsets.nbytes + res.supports.nbytes
        e2e_t = max_over_ranks(statistics.mean(e2e_ms))
        e2e = {"value": replicas.job_throughput(ref_supports, e2e_t, world), "unit": "supports/s",
               "h2d_bytes_per_step": int(h2d_bytes), "d2h_bytes_per_step": int(d2h), "ms_per_step": e2e_t,
               "steps": len(e2e_ms),
               "phases_ms": {k: statistics.mean(v) for k, v in ph.items()},
               "mine_path_ms": [statistics.mean(x[q] for x in first_paths) for q in range(len(first_paths[0]))],
               "timing": "host wall clock around open (H2D of the pinned CSR + device ingest) + mine (search, MFI "
                         "read-back into host memory) + close"}
        if plain_ms is not None:
            # the plain engine end to end: the same open and close around its mine
            e2e["plain_ms_per_step"] = e2e["phases_ms"]["open_ms"] + plain_ms + e2e["phases_ms"]["close_ms"]
            e2e["speedup_vs_plain"] = e2e["plain_ms_per_step"] / e2e_t

    # roofline per counting path over the timed steps
    traffic = None
    tp = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(tp):
        with open(tp) as f:
            traffic = json.load(f).get(args.workload)
    sm_mhz = (clk or {}).get("sm_mhz") or 1965.0
    paths = measure.path_rooflines(stats, pk["hbm_gbs"], i8_macs, sm_mhz=sm_mhz, sm_count=sm_count, traffic=traffic)
    roofline = measure.headline_roofline(paths, pk["hbm_gbs"], i8_macs, pk_src, i8_src)

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

    gpu_launches = int(sum(s["launches"] for s in stats))
    mean_stats = {k: (statistics.mean(s[k] for s in stats) if not isinstance(stats[0][k], list)
                      else [statistics.mean(s[k][q] for s in stats) for q in range(len(stats[0][k]))])
                  for k in stats[0]}
    out = {
        "metric": METRIC,
        "value": value, "unit": "supports/s", "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic",
        "config": {"workload": args.workload, "desc": w["desc"], "minsup": w["minsup"], "rows": db0.n_rows,
                   "reduced_rows": info["trans_num_reduced"], "survivors": info["n_survivors"],
                   "bitmap_bytes": int(info["n_dense"]) * int(info["words_per_row"]) * 4,
                   "l2": "inputs larger than L2 (bitmap) and a 256 MB L2 flush before every timed step",
                   "engine": args.engine, "counter": args.counter, "lookahead": args.lookahead,
                   "graphs": bool(args.graphs), "parallelism": f"{world} independent database replicas, one per GPU"},
        "value_basis": "reference-equivalent supports (the reference search's nodes x survivors, counted by the plain "
                       "engine) per second of batched mine time",
        "counted_supports_per_s": replicas.job_throughput(counted, ms, world),
        "reference_supports_per_db": ref_supports,
        "reference_supports_expected": w["ref_supports"],
        "counted_supports_per_db": counted,
        "mine_time_s": ms / 1000.0,
        "plain_mine_time_s": plain_ms / 1000.0 if plain_ms else None,
        "plain_runs": args.plain_runs if plain_ms else 0,
        "speedup_vs_plain": (plain_ms / ms) if plain_ms else None,
        "set_identical_to_plain": identical,
        "set_identical_to_reference_fixture": ident_gold,
        "n_mfi": len(batched),
        "stats": mean_stats,
        "plain_stats": plain.stats if plain else None,
        "roofline": roofline,
        "paths": paths,
        "peaks": {"hbm_gbs": pk["hbm_gbs"], "hbm_source": pk_src, "i8_macs_per_s": i8_macs, "i8_source": i8_src,
                  "popc_bitops_per_s": measure.popc_ceiling(sm_count, sm_mhz)},
        "ablation": ablation,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": gpu_launches,
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(out))
    if world > 1:
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
