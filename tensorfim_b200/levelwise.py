"""All frequent itemsets at the reference prototype's shape, on one GPU.

    python -m tensorfim_b200.levelwise [--tx 8388608] [--items 512] [--patterns 80]
                                       [--minsup 0.15] [--max-len 8] [--counter auto] [--seed 0]

The shape follows the reference's level-wise prototype (code/batch_proto/batch_proto.cu:45-52,
195-230): N transactions x d items as vertical bitmaps, planted patterns of 2..6 items that
fire i.i.d. per transaction with probability 0.2%..1.5%, light noise (0.02% of the
transactions per item), minimum support in percent of N, search up to 8 items.  The data
here is drawn from numpy's PCG64 with the given seed (not the prototype's generator).  The
mine runs through Database.mine_all (tfim_mine_all); the prototype's checks follow:
downward closure of the result and planted recall (a pattern is reported iff its exact
support, recomputed on the host, reaches the minimum).
"""
from __future__ import annotations

import argparse
import itertools
import json
import time

import numpy as np

from .engine import Database


def generate(n_tx: int, n_items: int, n_pat: int, seed: int = 0, max_pat: int = 6):
    rng = np.random.Generator(np.random.PCG64(seed))
    words = (n_tx + 31) // 32
    rows = np.zeros((n_items, words), np.uint32)
    pats = []

    def set_bits(item, t):
        np.bitwise_or.at(rows[item], t // 32, np.left_shift(np.uint32(1), (t % 32).astype(np.uint32)))

    for _ in range(n_pat):
        size = int(rng.integers(2, max_pat + 1))
        items = sorted(int(x) for x in rng.choice(n_items, size=size, replace=False))
        freq = (0.2 + 1.3 * rng.random()) / 100.0
        t = np.nonzero(rng.random(n_tx) < freq)[0]
        for it in items:
            set_bits(it, t)
        pats.append(items)
    for it in range(n_items):
        set_bits(it, rng.integers(0, n_tx, size=int(n_tx * 0.0002)))
    return rows, pats


def support(rows: np.ndarray, items) -> int:
    m = np.bitwise_and.reduce(rows[list(items)], axis=0)
    return int(np.unpackbits(m.view(np.uint8)).sum())


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--tx", type=int, default=1 << 23)
    ap.add_argument("--items", type=int, default=512)
    ap.add_argument("--patterns", type=int, default=80)
    ap.add_argument("--minsup", type=float, default=0.15, help="percent of the transactions")
    ap.add_argument("--max-len", type=int, default=8)
    ap.add_argument("--counter", default="auto")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--repeat", type=int, default=3)
    a = ap.parse_args()
    t0 = time.time()
    rows, pats = generate(a.tx, a.items, a.patterns, a.seed)
    gen_s = time.time() - t0
    min_count = int(a.tx * a.minsup / 100.0)
    with Database.from_bitmap(rows, a.tx, a.items) as db:
        db.set_counter(a.counter)
        best = None
        for _ in range(a.repeat):
            r = db.mine_all(min_count=min_count, max_len=a.max_len)
            if best is None or r.stats["mine_seconds"] < best.stats["mine_seconds"]:
                best = r
    found = {tuple(k): v for k, v in best.mfis}
    closed = all(sub in found for items in found if len(items) > 1
                 for sub in itertools.combinations(items, len(items) - 1))
    recalled = missed = false_pos = 0
    for p in pats:
        s = support(rows, p)
        inside = tuple(p) in found
        recalled += inside and s >= min_count
        missed += (not inside) and s >= min_count
        false_pos += inside and s < min_count
    levels = {}
    for k in found:
        levels[len(k)] = levels.get(len(k), 0) + 1
    print(json.dumps({"tx": a.tx, "items": a.items, "patterns": a.patterns, "min_count": min_count,
                      "max_len": a.max_len, "counter": a.counter, "itemsets": len(found), "per_level": levels,
                      "mine_seconds": best.stats["mine_seconds"], "count_kernel_ms": best.stats["kernel_ms"],
                      "waves": best.stats["waves"], "prefixes_counted": best.stats["nodes"],
                      "bitops_per_s": best.stats["bit_ops"] / max(best.stats["kernel_ms"] * 1e-3, 1e-12),
                      "downward_closure": closed, "planted": {"recalled": recalled, "missed": missed,
                                                              "false_positive": false_pos},
                      "generation_seconds": round(gen_s, 1)}))


if __name__ == "__main__":
    main()
