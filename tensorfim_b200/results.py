"""Results-file reading and comparison with the reference drivers' rules.

The drivers parse MFI lines with one regex (scripts/run_all_configs.py:27,
scripts/verify_all.py:13) and compare ``{frozenset(items): frequency}`` dicts for exact
equality (scripts/verify_all.py:39-45); header keys are read as ``key: value`` lines
(scripts/run_all_configs.py:25-26).
"""
from __future__ import annotations

import re

LINE = re.compile(r"^\d+th:\s+\d+\s+\{\s*([^}]*)\}\s+support:\s+\S+\s+frequency:\s+(\d+)")
KEY = re.compile(r"^([A-Za-z_()]+):\s*(\S+)")


def load_results(path: str) -> dict:
    sets = {}
    with open(path, encoding="utf-8", errors="replace") as f:
        for ln in f:
            m = LINE.match(ln.strip())
            if m:
                sets[frozenset(int(x) for x in m.group(1).split())] = int(m.group(2))
    return sets


def load_header(path: str) -> dict:
    out = {}
    with open(path, encoding="utf-8", errors="replace") as f:
        for ln in f:
            if LINE.match(ln.strip()):
                continue
            m = KEY.match(ln.strip())
            if m and m.group(1) not in out:
                out[m.group(1)] = m.group(2)
    return out


def compare(a: dict, b: dict) -> dict:
    """Set and frequency comparison of two MFI dicts."""
    ka, kb = set(a), set(b)
    return {
        "identical": a == b,
        "only_a": sorted(tuple(sorted(x)) for x in ka - kb)[:10],
        "only_b": sorted(tuple(sorted(x)) for x in kb - ka)[:10],
        "freq_mismatch": sorted((tuple(sorted(x)), a[x], b[x]) for x in ka & kb if a[x] != b[x])[:10],
        "n_a": len(a),
        "n_b": len(b),
    }
