"""One mine of a seeded benchmark database, for profiler captures.

    python -m tensorfim_b200.profcase --cfg 4 --scale 0.25 --counter tensor [--engine batched|resident|plain]
                                      [--top auto|bitmap|pairs] [--lookahead off|filtered|learned|all]
                                      [--graphs] [--repeat N] [--minsup F] [--replicas R]

Generates the configuration's database (tensorfim_b200.synth) at the given row scale,
builds it on cuda:0 and mines it once; prints the MFI count and the engine statistics.
"""
import argparse
import json

from . import synth
from .engine import Database

MINSUP = {1: 0.10, 2: 0.90, 3: 0.85, 4: 0.0005, 5: 0.70}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--cfg", type=int, default=4)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--minsup", type=float, default=None)
    ap.add_argument("--engine", default="batched")
    ap.add_argument("--counter", default="auto")
    ap.add_argument("--top", default="auto")
    ap.add_argument("--lookahead", default="learned", choices=["off", "filtered", "learned", "all"])
    ap.add_argument("--repeat", type=int, default=1)
    ap.add_argument("--graphs", action="store_true", help="resident engine: wave loop as a CUDA graph")
    ap.add_argument("--replicas", type=int, default=1, help="configuration 3: exact replicas of the base rows")
    a = ap.parse_args()
    kw = {"scale": a.scale} if a.cfg != 3 else {"scale": a.scale, "replicas": a.replicas}
    db0 = synth.generate(a.cfg, **kw)
    minsup = a.minsup if a.minsup is not None else MINSUP[a.cfg]
    with Database.from_csr(db0.offsets, db0.items, minsup) as db:
        for _ in range(a.repeat):
            r = db.mine(engine=a.engine, counter=a.counter, top=a.top, lookahead=a.lookahead, graphs=a.graphs)
        print(json.dumps({"mfis": len(r.mfis), "info": db.info, "stats": r.stats}))


if __name__ == "__main__":
    main()
