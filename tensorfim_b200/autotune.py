"""Autotuner: measures the engine's launch-shape and counter-selection parameters on the
GPU and writes the tuning table the library loads (tensorfim_b200/tuning.json).

    python -m tensorfim_b200.autotune [--out PATH] [--reps 5] [--quick]

Parameters (the tfim_tuning table of include/tfim.h):
  * wave_rows, l3_slices_per_sm, l3_dense_slices_per_sm, b1_tiles_per_sm, b1_min
    (b1_min_rows = b1_min_cols): coordinate descent over a grid, objective = the sum over the
    benchmark databases (configurations 1, 4 and 5 of tensorfim_b200.synth with their minimum
    supports, configuration 4 at 25% of its rows, and the dense replicated configuration at
    64 replicas with minsup 6%) of the median resident mine time with the learned proposal;
  * rate_b1_bitops, rate_lop3_bitops, rate_i8_bitops: bit-ops/s of one 256-node x 512-item
    counting wave over a random half-dense bitmap of 2^18 transactions, each counter forced
    (tensorfim_b200.countbench);
  * i8_min_rows = i8_min_cols: the square wave size from which the tcgen05 kind::i8 counter
    beats the b1 counter (waves of m x m over 2^20 transactions);
  * rate_pair_incr: pair increments/s of the empty-prefix family counted by pair
    co-occurrence on configuration 4 (sum over reduced rows of len^2/2 over its time).
Every mine of the sweep is checked against the first one: the table changes speed, never
the MFI set.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import time

import numpy as np

from . import synth
from .engine import Database, load_tuning, set_tuning, tuning

HERE = os.path.dirname(os.path.abspath(__file__))
TABLE = os.path.join(HERE, "tuning.json")

DATABASES = [("cfg4", 4, {}, 0.0005), ("cfg4_s025", 4, {"scale": 0.25}, 0.0005), ("cfg1", 1, {}, 0.10),
             ("cfg5", 5, {}, 0.70), ("dense_r64", 3, {"replicas": 64}, 0.06)]
GRID = {
    "wave_rows": [1024, 2048, 4096, 8192, 16384],
    "l3_slices_per_sm": [4.0, 8.0, 16.0, 32.0],
    "l3_dense_slices_per_sm": [32.0, 64.0, 128.0, 192.0],
    "b1_tiles_per_sm": [2.0, 4.0, 8.0, 16.0],
    "b1_min": [8, 16, 32, 64],
}


def _apply(params: dict) -> None:
    kw = dict(params)
    if "b1_min" in kw:
        m = kw.pop("b1_min")
        kw["b1_min_rows"] = kw["b1_min_cols"] = int(m)
    set_tuning(**kw)


def _objective(dbs, reps: int, ref: dict) -> tuple[float, dict]:
    per = {}
    for name, db in dbs:
        ts = []
        for _ in range(reps):
            r = db.mine(engine="resident", lookahead="learned")
            ts.append(r.stats["device_ms"])
            assert r.as_dict() == ref[name], f"tuning changed the MFI set of {name}"
        per[name] = statistics.median(ts)
    return sum(per.values()), per


def _bit_rates(reps: int) -> dict:
    from . import countbench
    r = countbench.run(256, 512, 1 << 18, counters=("tensor", "lop3", "i8"), reps=reps)["counters"]
    return {"rate_b1_bitops": r["tensor"]["bitops_per_s"], "rate_lop3_bitops": r["lop3"]["bitops_per_s"],
            "rate_i8_bitops": r["i8"]["bitops_per_s"]}


def _i8_crossover(reps: int) -> tuple[int, list]:
    """Smallest square wave size m (b = d = m nodes x items, 2^20 transactions) from which the
    tcgen05 kind::i8 counter beats the b1 counter at every larger size measured."""
    from . import countbench
    rec = []
    for m in (32, 64, 96, 128, 192, 256, 384):
        r = countbench.run(m, m, 1 << 20, counters=("tensor", "i8"), reps=reps)["counters"]
        rec.append([m, r["tensor"]["seconds"], r["i8"]["seconds"]])
    best = rec[-1][0] * 2
    for m, t_b1, t_i8 in reversed(rec):
        if t_i8 < t_b1:
            best = m
        else:
            break
    return best, rec


def _pair_rate(reps: int) -> float:
    db0 = synth.generate(4)
    minsup = 0.0005
    with Database.from_csr(db0.offsets, db0.items, minsup) as db:
        minc = db.info["min_count"]
        ts = [db.mine(engine="resident", top="pairs", lookahead="off").stats["top_ms"] for _ in range(reps)]
    freq = np.bincount(db0.items)
    keep = freq[db0.items] >= minc
    row = np.repeat(np.arange(db0.n_rows), np.diff(db0.offsets))
    lens = np.bincount(row[keep], minlength=db0.n_rows).astype(np.float64)
    work = float((lens * lens).sum()) / 2.0
    return work / (statistics.median(ts) / 1000.0)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=TABLE)
    ap.add_argument("--reps", type=int, default=5)
    ap.add_argument("--quick", action="store_true", help="two databases, three repetitions")
    a = ap.parse_args()
    reps = 3 if a.quick else a.reps
    t0 = time.time()
    start = tuning()
    dbs = []
    for name, cfg, kw, minsup in (DATABASES[:2] if a.quick else DATABASES):
        db0 = synth.generate(cfg, **kw)
        dbs.append((name, Database.from_csr(db0.offsets, db0.items, minsup)))
    ref = {name: db.mine(engine="resident", lookahead="learned").as_dict() for name, db in dbs}
    for _, db in dbs:   # warm-up
        db.mine(engine="resident", lookahead="learned")

    best = {"wave_rows": start["wave_rows"], "l3_slices_per_sm": start["l3_slices_per_sm"],
            "l3_dense_slices_per_sm": start["l3_dense_slices_per_sm"],
            "b1_tiles_per_sm": start["b1_tiles_per_sm"], "b1_min": start["b1_min_rows"]}
    _apply(best)
    best_obj, _ = _objective(dbs, reps, ref)
    sweeps = {}
    for key, values in GRID.items():
        rec = []
        for v in values:
            trial = dict(best, **{key: v})
            _apply(trial)
            obj, per = _objective(dbs, reps, ref)
            rec.append([v, round(obj, 4)] + [round(per[n], 4) for n, _ in dbs])
            if obj < best_obj * 0.98:   # keep a change only when it is clearly faster
                best, best_obj = trial, obj
        sweeps[key] = rec
        _apply(best)
    rates = _bit_rates(reps)
    rates["rate_pair_incr"] = _pair_rate(reps)
    i8_min, i8_rec = _i8_crossover(reps)
    for _, db in dbs:
        db.close()

    table = {"wave_rows": int(best["wave_rows"]), "l3_slices_per_sm": float(best["l3_slices_per_sm"]),
             "b1_tiles_per_sm": float(best["b1_tiles_per_sm"]), "b1_min_rows": int(best["b1_min"]),
             "b1_min_cols": int(best["b1_min"]), "proj_auto": int(start["proj_auto"]),
             "rate_b1_bitops": float(rates["rate_b1_bitops"]), "rate_lop3_bitops": float(rates["rate_lop3_bitops"]),
             "rate_pair_incr": float(rates["rate_pair_incr"]), "i8_min_rows": int(i8_min), "i8_min_cols": int(i8_min),
             "rate_i8_bitops": float(rates["rate_i8_bitops"]),
             "l3_dense_slices_per_sm": float(best["l3_dense_slices_per_sm"])}
    for k in ("tc_min_work", "tc_min_density", "tc_tiles_per_sm", "gram_min_rows"):   # not swept here
        table[k] = start[k]
    import torch
    doc = dict(table)
    doc["measured_on"] = torch.cuda.get_device_name(0)
    doc["objective_ms"] = round(best_obj, 4)
    doc["databases"] = [n for n, _ in dbs]
    doc["sweep_columns"] = ["value", "sum_ms"] + [n for n, _ in dbs]
    for k, rec in sweeps.items():
        doc["sweep:" + k] = rec
    doc["sweep:i8_crossover"] = {"columns": ["m", "b1_seconds", "i8_seconds"], "rows": i8_rec}
    doc["seconds"] = round(time.time() - t0, 1)
    with open(a.out, "w") as f:
        json.dump(doc, f, indent=1)
    load_tuning(a.out)
    print(json.dumps(doc))


if __name__ == "__main__":
    main()
