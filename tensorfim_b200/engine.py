"""Python mirror of the engine's C ABI (include/tfim.h).

The reference exposes two boundaries: the engine command line (``<exe> <transaction file>
<minsup>`` -> ``<file>-<minsup %f>=Results.txt``, code/engine/src/kernel_bitmap.cu:796-910)
and its counting contract (``getResFrequencyCuda`` :451-536, ``batchCountBMMA``
code/engine/src/kernel_bmma.cu:772-872).  ``mine_file`` runs the first through the
``tfim`` binary; ``Database.count_wave`` is the second; ``Database.mine`` is the search.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import _lib
from ._lib import TfimError, check, lib

ENGINES = {"plain": _lib.ENGINE_PLAIN, "batched": _lib.ENGINE_BATCHED, "resident": _lib.ENGINE_RESIDENT}
COUNTERS = {"auto": _lib.COUNTER_AUTO, "lop3": _lib.COUNTER_LOP3, "tensor": _lib.COUNTER_TENSOR,
            "proj": _lib.COUNTER_PROJ, "i8": _lib.COUNTER_I8}


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data) if a.size else C.c_void_p(0)


def _byte_view(data) -> np.ndarray:
    if isinstance(data, np.ndarray):
        return np.ascontiguousarray(data).view(np.uint8).reshape(-1)
    return np.frombuffer(memoryview(data), dtype=np.uint8)


def parse_text(data, device: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """The CSR (offsets int64, items int32) of a transaction file's bytes, parsed on the GPU
    with the reference's scanner rules (tfim_parse_text)."""
    buf = _byte_view(data)
    rows, n = C.c_int64(), C.c_int64()
    src = _ptr(buf) if buf.size else None
    check(lib().tfim_parse_text(src, buf.size, device, None, 0, None, 0, C.byref(rows), C.byref(n)))
    off = np.zeros(rows.value + 1, np.int64)
    items = np.zeros(max(n.value, 1), np.int32)
    check(lib().tfim_parse_text(src, buf.size, device, _ptr(off), off.size, _ptr(items), items.size, C.byref(rows),
                                C.byref(n)))
    return off, items[:n.value]


def read_fimi(path: str) -> tuple[np.ndarray, np.ndarray]:
    """Parse a transaction file with the reference's byte-scanner rules
    (code/engine/src/kernel_bitmap.cu:205-233): every '\\n' ends a row (empty rows
    included), digit runs are ids, a digit run right after '-' is dropped, every other
    byte separates, and a final row without '\\n' counts only when it holds an id.
    Returns CSR (offsets int64, items int32)."""
    buf = np.fromfile(path, dtype=np.uint8)
    n = buf.shape[0]
    if n == 0:
        return np.zeros(1, np.int64), np.zeros(0, np.int32)
    dig = (buf >= 48) & (buf <= 57)
    prev_dig = np.concatenate([[False], dig[:-1]])
    starts = np.flatnonzero(dig & ~prev_dig)
    nxt_dig = np.concatenate([dig[1:], [False]])
    ends = np.flatnonzero(dig & ~nxt_dig) + 1
    neg = np.zeros(starts.shape, dtype=bool)
    has_prev = starts > 0
    neg[has_prev] = buf[starts[has_prev] - 1] == 45
    lens = ends - starts
    vals = np.zeros(starts.shape, dtype=np.int64)
    for k in range(int(lens.max()) if lens.size else 0):
        m = lens > k
        vals[m] = vals[m] * 10 + (buf[starts[m] + k].astype(np.int64) - 48)
    nl = np.flatnonzero(buf == 10)
    keep = ~neg
    tok_row = np.searchsorted(nl, starts[keep], side="left")   # number of newlines before the token
    items = vals[keep].astype(np.int32)   # (int)long, as the reference
    n_rows = nl.shape[0]
    if tok_row.size and tok_row[-1] == n_rows:   # tokens after the last newline form a final row
        n_rows += 1
    counts = np.bincount(tok_row, minlength=n_rows)
    offsets = np.zeros(n_rows + 1, dtype=np.int64)
    offsets[1:] = np.cumsum(counts)
    return offsets, items


class MineResult:
    """The MFIs of one mine as flat arrays (``items[offsets[k]:offsets[k+1]]`` are the
    original ids of MFI k, largest first; ``supports[k]`` its support), in the order
    tfim_get_mfis returns them.  ``mfis`` builds the list of (items tuple, support) pairs
    on first use."""

    def __init__(self, items: np.ndarray, offsets: np.ndarray, supports: np.ndarray, stats: dict):
        self.items, self.offsets, self.supports, self.stats = items, offsets, supports, stats
        self._mfis = None

    def __len__(self) -> int:
        return int(self.supports.shape[0])

    @property
    def mfis(self) -> list:
        if self._mfis is None:
            it, off = self.items.tolist(), self.offsets.tolist()
            self._mfis = [(tuple(it[off[k]:off[k + 1]]), s) for k, s in enumerate(self.supports.tolist())]
        return self._mfis

    def as_dict(self) -> dict:
        return {frozenset(items): sup for items, sup in self.mfis}


def tuning() -> dict:
    """The tuning table in force (include/tfim.h tfim_tuning)."""
    t = _lib.Tuning()
    lib().tfim_tuning_get(C.byref(t))
    return t.as_dict()


def set_tuning(**values) -> None:
    """Replace entries of the tuning table, e.g. set_tuning(wave_rows=2048)."""
    t = _lib.Tuning()
    lib().tfim_tuning_get(C.byref(t))
    for k, v in values.items():
        if k not in t.as_dict():
            raise KeyError(k)
        setattr(t, k, v)
    check(lib().tfim_tuning_set(C.byref(t)))


def load_tuning(path: str) -> None:
    check(lib().tfim_tuning_load(path.encode()))


def tuning_source() -> str:
    return lib().tfim_tuning_source().decode()


_SHIPPED = {}


def shipped_proposal(device: int = 0):
    """The trained proposal network shipped with the package, loaded once per device and
    shared by every Database on that device (a context does not own its proposal)."""
    if device not in _SHIPPED:
        from .learn import Proposal
        _SHIPPED[device] = Proposal.load(device=device)
    return _SHIPPED[device]


class Database:
    """A transaction database resident on one GPU (a tfim_ctx)."""

    def __init__(self, handle: C.c_void_p, device: int = 0, group=None):
        self._h = handle
        self._device = device
        self._proposal = None
        self._group = group   # a sharded context calls back into it: kept alive while open
        self.sharded = group is not None
        info = _lib.DbInfo()
        check(lib().tfim_db_info_get(self._h, C.byref(info)))
        self.info = info.as_dict()

    # -- construction ------------------------------------------------------------------
    @classmethod
    def from_csr(cls, offsets: np.ndarray, items: np.ndarray, minsup: float, device: int = 0) -> "Database":
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        items = np.ascontiguousarray(items, dtype=np.int32)
        h = C.c_void_p()
        check(lib().tfim_open_db(_ptr(offsets), _ptr(items), offsets.shape[0] - 1, float(minsup), device, C.byref(h)))
        return cls(h, device)

    @classmethod
    def from_file(cls, path: str, minsup: float, device: int = 0) -> "Database":
        """A transaction file, read into pinned staging and parsed on the GPU (tfim_open_file)."""
        h = C.c_void_p()
        check(lib().tfim_open_file(os.fsencode(path), float(minsup), device, C.byref(h)))
        return cls(h, device)

    @classmethod
    def from_text(cls, data, minsup: float, device: int = 0) -> "Database":
        """The bytes of a transaction file (bytes, bytearray or a uint8 array, pinned or not),
        parsed on the GPU (tfim_open_text)."""
        buf = _byte_view(data)
        h = C.c_void_p()
        check(lib().tfim_open_text(_ptr(buf) if buf.size else None, buf.size, float(minsup), device, C.byref(h)))
        return cls(h, device)

    @classmethod
    def from_bitmap(cls, rows: np.ndarray, n_bits: int, n_counted: int, device: int = 0) -> "Database":
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        h = C.c_void_p()
        check(lib().tfim_open_bitmap(_ptr(rows), rows.shape[0], int(n_bits), int(n_counted), device, C.byref(h)))
        return cls(h, device)

    @classmethod
    def from_csr_sharded(cls, offsets: np.ndarray, items: np.ndarray, minsup: float, group, device: int = 0) -> "Database":
        """This shard's rows of a transaction-sharded database (tfim_open_db_sharded); `group` is
        a tensorfim_b200.shard.Group (TorchGroup, or a ThreadGroup member).  Counts, info and
        mined sets are the whole database's; every shard must make the same calls."""
        offsets = np.ascontiguousarray(offsets, dtype=np.int64)
        items = np.ascontiguousarray(items, dtype=np.int32)
        g = group.struct()
        h = C.c_void_p()
        check(lib().tfim_open_db_sharded(_ptr(offsets), _ptr(items), offsets.shape[0] - 1, float(minsup), device,
                                         C.byref(g), C.byref(h)))
        return cls(h, device, group)

    @classmethod
    def from_bitmap_sharded(cls, rows: np.ndarray, n_bits: int, n_counted: int, group, device: int = 0) -> "Database":
        """This shard's transactions (bit columns) of a vertical bitmap (tfim_open_bitmap_sharded)."""
        rows = np.ascontiguousarray(rows, dtype=np.uint32)
        g = group.struct()
        h = C.c_void_p()
        check(lib().tfim_open_bitmap_sharded(_ptr(rows), rows.shape[0], int(n_bits), int(n_counted), device,
                                             C.byref(g), C.byref(h)))
        return cls(h, device, group)

    # -- tables --------------------------------------------------------------------------
    def dense_to_orig(self) -> np.ndarray:
        out = np.zeros(self.info["n_dense"], dtype=np.int32)
        check(lib().tfim_dense_to_orig(self._h, _ptr(out)))
        return out

    def dense_freq(self) -> np.ndarray:
        out = np.zeros(self.info["n_dense"], dtype=np.int32)
        check(lib().tfim_dense_freq(self._h, _ptr(out)))
        return out

    # -- counting contract ---------------------------------------------------------------
    def count_wave(self, lists: list, min_count: int, counter: str = "auto") -> tuple[np.ndarray, np.ndarray]:
        """Supports of every counted item against each node's prefix (AND of its dense
        item list): counts[i, e] and nfreq[i] = #{e : counts[i, e] >= min_count}."""
        b = len(lists)
        d = self.info["n_survivors"]
        offs = np.zeros(b + 1, dtype=np.int64)
        offs[1:] = np.cumsum([len(x) for x in lists])
        flat = np.array([x for l in lists for x in l], dtype=np.int32)
        counts = np.zeros((b, d), dtype=np.int32)
        nfreq = np.zeros(b, dtype=np.int32)
        check(lib().tfim_set_counter(self._h, COUNTERS[counter]))
        check(lib().tfim_count_wave(self._h, _ptr(flat), _ptr(offs), b, int(min_count), _ptr(counts), _ptr(nfreq)))
        return counts, nfreq

    def set_counter(self, counter: str) -> None:
        """Counter used by count_wave / count_wave_device: auto, lop3, tensor."""
        check(lib().tfim_set_counter(self._h, COUNTERS[counter]))

    def count_wave_device(self, d_items: int, d_offsets: int, b: int, max_len: int, min_count: int,
                          d_counts: int, d_nfreq: int, stream: int = 0) -> None:
        """Device-pointer form (e.g. torch tensors' data_ptr()), ordered on `stream`."""
        check(lib().tfim_count_wave_device(self._h, C.c_void_p(d_items), C.c_void_p(d_offsets), int(b), int(max_len),
                                           int(min_count), C.c_void_p(d_counts), C.c_void_p(d_nfreq),
                                           C.c_void_p(stream or None)))

    # -- search ----------------------------------------------------------------------------
    def set_proposal(self, proposal, threshold: float | None = None) -> None:
        """Attach a learned lookahead proposal (tensorfim_b200.learn.Proposal) or None."""
        self._proposal = proposal   # keep it alive while attached
        h = proposal._h if proposal is not None else None
        thr = threshold if threshold is not None else (proposal.threshold if proposal is not None else 0.5)
        check(lib().tfim_set_proposal(self._h, h, float(thr)))

    def lookahead_log(self) -> tuple[np.ndarray, np.ndarray]:
        """Features (n x 32) and outcomes of the lookaheads logged by the last mine."""
        n = lib().tfim_lookahead_log(self._h, None, None, 0)
        if n < 0:
            raise TfimError(-n, lib().tfim_last_error().decode())
        x = np.zeros((n, 32), np.float32)
        y = np.zeros(n, np.float32)
        if n:
            lib().tfim_lookahead_log(self._h, _ptr(x), _ptr(y), n)
        return x, y

    def mine(self, engine: str | None = None, counter: str = "auto", lookahead=True,
             wave_cap: int = 0, top: str = "auto", log_lookahead: bool = False, proj_auto: int = -1,
             graphs: bool = False, small_pools: bool = False, superset: bool = False) -> MineResult:
        """lookahead: False/"off", True/"filtered" (every node passing the exact tail-pair
        filter), "learned" (the attached proposal, or the shipped weights), "all".
        graphs: (resident engine) run the wave loop as a captured CUDA graph whose conditional
        WHILE node repeats pack -> count -> expand on the device; the host reads the status
        only when the search ends or a pool has to grow.
        superset: (resident engine) drop a family whose head and tail lie inside an MFI already
        found; the MFI set is the same either way (off by default: it found nothing to drop
        on the benchmark databases and costs 3-10% of the mine time).
        engine: "resident" (default), "batched" (default for a sharded database) or "plain"."""
        o = _lib.MineOpts()
        lib().tfim_mine_opts_default(C.byref(o))
        o.engine = ENGINES[engine or ("batched" if self.sharded else "resident")]
        o.counter = COUNTERS[counter]
        la = {False: 0, True: 1, "off": 0, "filtered": 1, "learned": 2, "all": 3}[lookahead]
        if la == 2 and getattr(self, "_proposal", None) is None:
            self.set_proposal(shipped_proposal(self._device))
        o.lookahead = la
        o.log_lookahead = int(log_lookahead)
        o.proj_auto = int(proj_auto)
        o.wave_cap = int(wave_cap)
        o.top_counter = {"auto": 0, "bitmap": 1, "pairs": 2}[top]
        o.use_graphs = int(bool(graphs))
        o.small_pools = int(bool(small_pools))
        o.superset = int(bool(superset))
        st = _lib.MineStats()
        check(lib().tfim_mine(self._h, C.byref(o), C.byref(st)))
        n = lib().tfim_num_mfis(self._h)
        tot = lib().tfim_mfi_item_total(self._h)
        items = np.zeros(max(tot, 1), dtype=np.int32)
        offs = np.zeros(n + 1, dtype=np.int64)
        sup = np.zeros(max(n, 1), dtype=np.int32)
        check(lib().tfim_get_mfis(self._h, _ptr(items), _ptr(offs), _ptr(sup)))
        return MineResult(items[:tot], offs, sup[:n], st.as_dict())

    def mine_all(self, min_count: int | None = None, max_len: int = 8, max_itemsets: int = 50_000_000) -> MineResult:
        """All frequent itemsets of up to max_len items (support >= min_count; default the
        database's minimum count), level by level on the counting contract -- the reference's
        level-wise prototype (code/batch_proto/batch_proto.cu).  Items in original ids,
        in ascending dense-id order; singletons carry their bitmap support."""
        mc = int(self.info["min_count"] if min_count is None else min_count)
        st = _lib.MineStats()
        check(lib().tfim_mine_all(self._h, mc, int(max_len), int(max_itemsets), C.byref(st)))
        n = lib().tfim_num_all(self._h)
        tot = lib().tfim_all_item_total(self._h)
        items = np.zeros(max(tot, 1), dtype=np.int32)
        offs = np.zeros(n + 1, dtype=np.int64)
        sup = np.zeros(max(n, 1), dtype=np.int32)
        check(lib().tfim_get_all(self._h, _ptr(items), _ptr(offs), _ptr(sup)))
        return MineResult(items[:tot], offs, sup[:n], st.as_dict())

    def write_results(self, trans_set_file: str, result_path: str, prep_s: float = 0.0, comp_s: float = 0.0) -> None:
        check(lib().tfim_write_results(self._h, trans_set_file.encode(), result_path.encode(), prep_s, comp_s))

    def close(self) -> None:
        if self._h:
            lib().tfim_close(self._h)
            self._h = None
        self._proposal = None
        self._group = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def release_cached(device: int = -1) -> None:
    """Free the device pools closed databases left for the next one (tfim_release_cached),
    on `device` or on every device."""
    check(lib().tfim_release_cached(int(device)))


def result_path(path: str, minsup: float) -> str:
    """The reference's result-file name: sprintf("%s-%f=Results.txt") (kernel_bitmap.cu:906-907)."""
    return "%s-%f=Results.txt" % (path, minsup)


def mine_file(path: str, minsup: float, engine: str = "resident", counter: str = "auto", lookahead: int = 1,
              timeout: float | None = None, graphs: bool = False) -> subprocess.CompletedProcess:
    """Run the `tfim` command-line engine exactly as a driver runs the reference's exe."""
    if not os.path.exists(_lib.CLI_PATH):
        raise TfimError(-1, f"{_lib.CLI_PATH} is missing: build it with `python -m tensorfim_b200.build`")
    cmd = [_lib.CLI_PATH, path, repr(float(minsup)), "--engine", engine, "--counter", counter,
           "--lookahead", str(int(lookahead)), "--graphs", str(int(bool(graphs)))]
    return subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
