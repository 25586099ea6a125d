"""Python access to the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only tests/, __graft_entry__.smoke() (as the checker) and bench.py's CPU-baseline leg
may use this module.  It wraps
  * _build/liboracle.so: tfim_oracle.c, the C restatement of the reference engine;
  * _ref/tfim_ref_*: the reference engine compiled from its own sources (oracle/Makefile),
    present when the reference tree was available at build time.
"""
from __future__ import annotations

import ctypes as C
import os
import re
import shutil
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "_build", "liboracle.so")
REF_DIR = os.path.join(HERE, "_ref")
REF_SERIAL = os.path.join(REF_DIR, "tfim_ref_serial")
REF_MT = os.path.join(REF_DIR, "tfim_ref_mt")
REF_GPU = os.path.join(REF_DIR, "tfim_ref_gpu")
REF_BMMA = os.path.join(REF_DIR, "tfim_ref_bmma")
# the reference project checkout the _ref binaries are compiled from (read in place)
REFERENCE_TREE = os.environ.get("TFIM_REFERENCE", "/root/reference")

LINE = re.compile(r"^\d+th:\s+\d+\s+\{\s*([^}]*)\}\s+support:\s+\S+\s+frequency:\s+(\d+)")


def build(reference_tree: str | None = None) -> None:
    """make the oracle (and, when the reference tree exists, the reference binaries)."""
    subprocess.run(["make", "-s", "-C", HERE, "all"], check=True)
    tree = reference_tree or REFERENCE_TREE
    if os.path.isdir(os.path.join(tree, "code", "engine", "src")):
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={tree}"], check=True)


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        p, i32, i64 = C.c_void_p, C.c_int32, C.c_int64
        L.tfo_load.restype = p
        L.tfo_load.argtypes = [C.c_char_p, C.c_double]
        L.tfo_load_csr.restype = p
        L.tfo_load_csr.argtypes = [p, p, i64, C.c_double]
        L.tfo_mine_sample.restype = i64
        L.tfo_mine_sample.argtypes = [p, C.c_double, C.c_int, C.POINTER(C.c_double)]
        L.tfo_free.argtypes = [p]
        L.tfo_mine.restype = i64
        L.tfo_mine.argtypes = [p, C.c_int]
        for name in ["tfo_num_mfis", "tfo_nodes_visited", "tfo_num_reduced", "tfo_num_trans",
                     "tfo_dimension_reduced", "tfo_mfi_item_total", "tfo_w64"]:
            getattr(L, name).restype = i64
            getattr(L, name).argtypes = [p]
        for name in ["tfo_num_survivors", "tfo_dcount"]:
            getattr(L, name).restype = i32
            getattr(L, name).argtypes = [p]
        L.tfo_comp_time.restype = C.c_double
        L.tfo_comp_time.argtypes = [p]
        L.tfo_frequency_threshold.restype = C.c_double
        L.tfo_frequency_threshold.argtypes = [p]
        L.tfo_get_mfis.argtypes = [p, p, p, p]
        L.tfo_bitmap.restype = p
        L.tfo_bitmap.argtypes = [p]
        for name in ["tfo_dense_to_orig", "tfo_freq_dense", "tfo_items_in_freq_sort"]:
            getattr(L, name).argtypes = [p, p]
        L.tfo_write_results.argtypes = [p, C.c_char_p, C.c_char_p]
        L.tfo_count_wave.argtypes = [p, i64, p, p, i32, i32, i32, p, p]
        L.tfo_parse.argtypes = [C.c_char_p, C.POINTER(i64), C.POINTER(i64), p, i64, p, i64]
        _lib = L
    return _lib


def _p(a):
    return C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(0)


class OracleDB:
    """A database parsed, reduced and bitmapped by the oracle from a transaction file."""

    def __init__(self, path: str | None, minsup: float, csr: tuple | None = None):
        self.path = path or "<memory>"
        self.minsup = minsup
        if csr is not None:
            off = np.ascontiguousarray(csr[0], dtype=np.int64)
            items = np.ascontiguousarray(csr[1], dtype=np.int32)
            self.h = lib().tfo_load_csr(_p(off), _p(items), off.shape[0] - 1, float(minsup))
        else:
            self.h = lib().tfo_load(path.encode(), float(minsup))
        if not self.h:
            raise FileNotFoundError(path)

    def mine_sample(self, budget_s: float, threads: int = 0) -> tuple[int, float]:
        """Nodes counted and seconds spent on a time-bounded sample of root subtrees."""
        secs = C.c_double()
        nodes = lib().tfo_mine_sample(self.h, float(budget_s), threads, C.byref(secs))
        return int(nodes), float(secs.value)

    def mine(self, threads: int = 0) -> dict:
        L = lib()
        L.tfo_mine(self.h, threads)
        n = L.tfo_num_mfis(self.h)
        tot = L.tfo_mfi_item_total(self.h)
        items = np.zeros(max(tot, 1), np.int32)
        offs = np.zeros(n + 1, np.int64)
        sup = np.zeros(max(n, 1), np.int32)
        L.tfo_get_mfis(self.h, _p(items), _p(offs), _p(sup))
        return {frozenset(int(x) for x in items[offs[k]:offs[k + 1]]): int(sup[k]) for k in range(n)}

    def mine_list(self, threads: int = 0) -> list:
        """MFIs as (items in print order, support), the reference's sort by support."""
        L = lib()
        L.tfo_mine(self.h, threads)
        n = L.tfo_num_mfis(self.h)
        tot = L.tfo_mfi_item_total(self.h)
        items = np.zeros(max(tot, 1), np.int32)
        offs = np.zeros(n + 1, np.int64)
        sup = np.zeros(max(n, 1), np.int32)
        L.tfo_get_mfis(self.h, _p(items), _p(offs), _p(sup))
        return [(tuple(int(x) for x in items[offs[k]:offs[k + 1]]), int(sup[k])) for k in range(n)]

    @property
    def nodes(self) -> int:
        return lib().tfo_nodes_visited(self.h)

    @property
    def comp_time(self) -> float:
        return lib().tfo_comp_time(self.h)

    def info(self) -> dict:
        L = lib()
        return {"n_survivors": L.tfo_num_survivors(self.h), "trans_num_reduced": L.tfo_num_reduced(self.h),
                "trans_num": L.tfo_num_trans(self.h), "dimension_reduced": L.tfo_dimension_reduced(self.h),
                "frequency_threshold": L.tfo_frequency_threshold(self.h), "n_dense": L.tfo_dcount(self.h)}

    def write_results(self, result_path: str) -> None:
        lib().tfo_write_results(self.h, self.path.encode(), result_path.encode())

    def close(self):
        if self.h:
            lib().tfo_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def mine_file(path: str, minsup: float, threads: int = 0) -> dict:
    db = OracleDB(path, minsup)
    try:
        return db.mine(threads)
    finally:
        db.close()


def parse_file(path: str) -> tuple[np.ndarray, np.ndarray]:
    """The oracle's parse of a transaction file as CSR (offsets int64, items int32)."""
    L = lib()
    rows, n = C.c_int64(), C.c_int64()
    if L.tfo_parse(path.encode(), C.byref(rows), C.byref(n), None, 0, None, 0) != 0:
        raise FileNotFoundError(path)
    off = np.zeros(rows.value + 1, np.int64)
    items = np.zeros(max(n.value, 1), np.int32)
    L.tfo_parse(path.encode(), C.byref(rows), C.byref(n), _p(off), off.size, _p(items), items.size)
    return off, items[:n.value]


def count_wave(rows: np.ndarray, lists: list, d: int, min_count: int) -> tuple[np.ndarray, np.ndarray]:
    """The counting contract on the CPU: rows is (n_rows, words) uint32."""
    rows = np.ascontiguousarray(rows, dtype=np.uint32)
    b = len(lists)
    offs = np.zeros(b + 1, np.int64)
    offs[1:] = np.cumsum([len(x) for x in lists])
    flat = np.array([x for l in lists for x in l], dtype=np.int32)
    counts = np.zeros((b, d), np.int32)
    nfreq = np.zeros(b, np.int32)
    lib().tfo_count_wave(_p(rows), rows.shape[1], _p(flat), _p(offs), b, d, int(min_count), _p(counts), _p(nfreq))
    return counts, nfreq


def load_results(path: str) -> dict:
    sets = {}
    with open(path, encoding="utf-8", errors="replace") as f:
        for ln in f:
            m = LINE.match(ln.strip())
            if m:
                sets[frozenset(int(x) for x in m.group(1).split())] = int(m.group(2))
    return sets


def run_reference(path: str, minsup: float, binary: str = REF_SERIAL, threads: int | None = None,
                  timeout: float = 600, in_place: bool = False, stdout: dict | None = None) -> tuple[dict, dict]:
    """Run a reference binary on a copy of `path` in a scratch directory (its results file
    is written next to its input), or on `path` itself with `in_place` (its directory must
    be writable; the results file is removed afterwards).  Returns (mfis, header); when
    `stdout` is a dict, its "text" gets the run's standard output and "wall_s" its wall time."""
    if not os.path.exists(binary):
        raise FileNotFoundError(binary)
    with tempfile.TemporaryDirectory() as d:
        if in_place:
            dst = path
        else:
            dst = os.path.join(d, os.path.basename(path))
            shutil.copyfile(path, dst)
        env = dict(os.environ)
        if threads:
            env["TFIM_REF_THREADS"] = str(threads)
            env["OMP_NUM_THREADS"] = str(threads)
        import time
        t0 = time.perf_counter()
        r = subprocess.run([binary, dst, "%r" % float(minsup)], capture_output=True, text=True, env=env,
                           timeout=timeout, cwd=os.path.dirname(os.path.abspath(dst)))
        if stdout is not None:
            stdout["text"] = r.stdout
            stdout["wall_s"] = time.perf_counter() - t0
        res = "%s-%f=Results.txt" % (dst, minsup)
        if not os.path.exists(res):
            raise RuntimeError(f"reference run produced no results file (rc={r.returncode}): {r.stdout[-500:]} {r.stderr[-500:]}")
        header = {}
        with open(res, errors="replace") as f:
            for ln in f:
                m = re.match(r"^([A-Za-z_()]+):\s*(\S+)", ln.strip())
                if m and m.group(1) not in header:
                    header[m.group(1)] = m.group(2)
        mfis = load_results(res)
        if in_place:
            os.unlink(res)
        return mfis, header
