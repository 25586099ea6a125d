"""Generate the golden fixtures of tests/golden/ by running the REFERENCE engine itself.

The reference engine (code/engine/src/kernel_bitmap.cu, serial RUN_MODE 0) is compiled
from its own sources by oracle/Makefile into oracle/_ref/tfim_ref_serial.  This script
runs it on
  * seeded synthetic databases of the benchmark shapes (tensorfim_b200.synth), at sizes
    the reference finishes in seconds -- the inputs are regenerated at test time from the
    same seeds, so only the expected outputs are stored;
  * small hand-made edge-case files (stored as <name>.txt beside their outputs): a
    frequent item 0, repeated ids within a row, empty lines / CRLF / negative ids /
    an unterminated last line, exact-threshold ties, a single row, identical rows, and
    a threshold no item reaches.
Each fixture <name>.json.gz holds the spec, the reference's header statistics and its MFIs
as [sorted item list, frequency] pairs.

Run from the repository root:  python tests/golden/make_golden.py [name ...]
(with names, only those fixtures are regenerated; the full-size fixtures of full/, minutes of
CPU each, only when named: python tests/golden/make_golden.py cfg5_full cfg4_full).
"""
from __future__ import annotations

import gzip
import json
import os
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle  # noqa: E402
from tensorfim_b200 import synth  # noqa: E402

SYNTH = [
    # name, config, generator kwargs, minsup
    ("cfg1_full", 1, {}, 0.10),
    ("cfg2_full", 2, {}, 0.90),
    ("cfg3_base", 3, {"replicas": 1}, 0.85),
    ("cfg3_base_t30", 3, {"replicas": 1, "scale": 0.2}, 0.30),
    ("cfg4_s001", 4, {"scale": 0.01}, 0.005),
    ("cfg5_s002", 5, {"scale": 0.02}, 0.70),
    ("cfg5_s002_t40", 5, {"scale": 0.02}, 0.40),
    ("cfg1_t03", 1, {"scale": 0.5}, 0.03),
    # the replicated 12.54M configuration's generator at its base size (1 replica) with the
    # minimum support lowered from 85% to 6% (at 85% no item is frequent); supports of the
    # 256-replica database are exactly 256x these
    ("cfg3_base_t06", 3, {"replicas": 1}, 0.06),
]


# Full-size databases of the benchmark shapes, stored under full/ (the per-variant fixture
# tests do not scan it): the reference's multithreaded CPU engine (the same kernel_bitmap.cu,
# RUN_MODE 2 with every node on its CPU counter, oracle/_ref/tfim_ref_mt) on all host threads.
FULL = [
    ("cfg5_full", 5, {}, 0.70),
    ("cfg4_full", 4, {}, 0.0005),
]


def edge_files() -> dict:
    """name -> (file bytes, minsup)."""
    out = {}
    # item 0 frequent and a root: the reference parks it after the survivors
    rows = []
    for r in range(200):
        row = [0] if r % 5 != 0 else []
        row += [1 + (r % 3), 4 + (r % 2), 7]
        if r % 7 == 0:
            row.append(9)
        rows.append(" ".join(map(str, row)))
    out["edge_item0"] = ("\n".join(rows) + "\n").encode(), 0.3
    # repeated ids inside rows: F1 counts occurrences, the bitmap counts rows
    rows = []
    for r in range(120):
        row = [1, 2, 3] if r % 2 else [2, 3, 3, 3]
        if r % 3 == 0:
            row += [5, 5, 6]
        if r % 4 == 0:
            row += [7, 1, 1]
        rows.append(" ".join(map(str, row)))
    out["edge_dups"] = ("\n".join(rows) + "\n").encode(), 0.4
    # empty lines, CRLF, tabs, negative ids, an unterminated last line
    txt = "1 2 3\r\n\n2 3 -4 5\n\t3 5 6\n\n1 -2 3 5\n2 3 5\n1 2 3 5\n3 5 x 6\n1 3 5"
    out["edge_format"] = txt.encode(), 0.25
    # exact-threshold ties: 100 rows at 0.2 -> 20.0; items at exactly 20 are extensions, not roots
    rows = []
    for r in range(100):
        row = [1]
        if r < 20:
            row.append(2)
        if r < 40:
            row.append(3)
        if 10 <= r < 30:
            row.append(4)
        if r % 2 == 0:
            row.append(5)
        rows.append(" ".join(map(str, row)))
    out["edge_ties"] = ("\n".join(rows) + "\n").encode(), 0.2
    out["edge_single"] = b"3 1 4 1 5 9 2 6\n", 1.0
    out["edge_identical"] = ("\n".join(["2 4 6 8"] * 50) + "\n").encode(), 0.5
    out["edge_none"] = ("\n".join(str(i) for i in range(1, 101)) + "\n").encode(), 0.5
    return out


def main(only: list[str]) -> None:
    if not os.path.exists(oracle.REF_SERIAL):
        oracle.build()
    with tempfile.TemporaryDirectory() as d:
        for name, cfg, kw, minsup in SYNTH:
            if only and name not in only:
                continue
            db = synth.generate(cfg, **kw)
            path = os.path.join(d, name + ".txt")
            synth.write_fimi(path, db)
            mfis, hdr = oracle.run_reference(path, minsup, timeout=1800)
            spec = {"kind": "synth", "config": cfg, "kwargs": kw, "minsup": minsup}
            _dump(name, spec, hdr, mfis)
        for name, cfg, kw, minsup in FULL:
            if name not in only:   # minutes each: only when named
                continue
            db = synth.generate(cfg, **kw)
            path = os.path.join(d, name + ".txt")
            synth.write_fimi(path, db)
            mfis, hdr = oracle.run_reference(path, minsup, binary=oracle.REF_MT, threads=os.cpu_count() or 1,
                                             timeout=7200)
            spec = {"kind": "synth", "config": cfg, "kwargs": kw, "minsup": minsup}
            _dump(name, spec, hdr, mfis, sub="full", generator="reference engine (kernel_bitmap.cu, RUN_MODE 2, "
                  "multithreaded CPU counter) built by oracle/Makefile")
        for name, (blob, minsup) in edge_files().items():
            if only and name not in only:
                continue
            path = os.path.join(HERE, name + ".txt")
            with open(path, "wb") as f:
                f.write(blob)
            mfis, hdr = oracle.run_reference(path, minsup)
            spec = {"kind": "file", "file": name + ".txt", "minsup": minsup}
            _dump(name, spec, hdr, mfis)


def _dump(name, spec, hdr, mfis, sub: str = "",
          generator: str = "reference engine (kernel_bitmap.cu, RUN_MODE 0) built by oracle/Makefile"):
    keep = ["transNum", "dimension", "itemIDmin", "itemIDmax", "transLengthMin", "transLengthMax", "transLengthMean",
            "dimensionReduced", "transNumReduced", "transLengthReducedMin", "transLengthReducedMax",
            "transLengthReducedMean", "MFIsNumber"]
    out = {
        "spec": spec,
        "generator": generator,
        "header": {k: hdr.get(k) for k in keep},
        "mfis": sorted([sorted(s), f] for s, f in mfis.items()),
    }
    os.makedirs(os.path.join(HERE, sub), exist_ok=True)
    with gzip.open(os.path.join(HERE, sub, name + ".json.gz"), "wt") as f:
        json.dump(out, f, separators=(",", ":"))
    print(f"{name}: {len(mfis)} MFIs")


if __name__ == "__main__":
    main(sys.argv[1:])
