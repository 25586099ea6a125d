"""Transaction sharding on the CPU: shard bounds, the all-reduce callback's status contract,
and -- on two gloo ranks -- the arithmetic the sharded library relies on: F1 counts and
prefix-by-item supports counted per shard (by the oracle) and summed over the group equal
the whole database's, while per-shard thresholds would not."""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

from tensorfim_b200 import _lib  # noqa: E402
from tensorfim_b200.shard import Group, shard_bounds, shard_csr  # noqa: E402


def test_shard_bounds_partition():
    for n in (0, 1, 5, 100, 1001):
        for world in (1, 2, 3, 7):
            b = [shard_bounds(n, r, world) for r in range(world)]
            assert b[0][0] == 0 and b[-1][1] == n
            assert all(b[r][1] == b[r + 1][0] for r in range(world - 1))
            sizes = [hi - lo for lo, hi in b]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def test_shard_csr_concatenates_to_the_whole():
    rng = np.random.default_rng(0)
    lens = rng.integers(0, 6, size=37)
    off = np.concatenate([[0], np.cumsum(lens)]).astype(np.int64)
    items = rng.integers(0, 20, size=off[-1]).astype(np.int32)
    for world in (1, 2, 5, 40):
        parts = [shard_csr(off, items, r, world) for r in range(world)]
        assert all(p[0][0] == 0 for p in parts)
        assert sum(p[0].shape[0] - 1 for p in parts) == 37
        np.testing.assert_array_equal(np.concatenate([p[1] for p in parts]), items)
        np.testing.assert_array_equal(np.concatenate([np.diff(p[0]) for p in parts]), lens)


class _Recorder(Group):
    def __init__(self, fail=False):
        super().__init__(0, 2)
        self.calls, self.fail = [], fail

    def allreduce(self, ptr, count, dtype, op, stream):
        if self.fail:
            raise RuntimeError("peer left")
        self.calls.append((ptr, count, dtype, op, stream))


def test_callback_status_contract():
    ok = _Recorder()
    st = ok.struct()
    assert (st.rank, st.world) == (0, 2)
    assert st.allreduce(4096, 12, _lib.DT_I64, _lib.RED_MAX, 77, None) == 0
    assert ok.calls == [(4096, 12, _lib.DT_I64, _lib.RED_MAX, 77)]
    bad = _Recorder(fail=True)
    assert bad.struct().allreduce(4096, 1, _lib.DT_I32, _lib.RED_SUM, None, None) == 1
    assert "peer left" in bad.last_error
    with pytest.raises(ValueError):
        Group(3, 2)


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _bitmap(off, items, dense_of, d):
    """Rows = dense items (0..d-1), columns = this shard's transactions."""
    n = off.shape[0] - 1
    w = max(1, (n + 31) // 32)
    bits = np.zeros((d, w * 32), bool)
    rows = np.repeat(np.arange(n), np.diff(off))
    dj = dense_of[items]
    keep = (dj >= 0) & (dj < d)
    bits[dj[keep], rows[keep]] = True
    return np.ascontiguousarray(np.packbits(bits, axis=1, bitorder="little").view("<u4"))


def _rank_main(rank, world, port, out_dir):
    import datetime

    import torch
    import torch.distributed as dist

    from oracle import oracle
    from tensorfim_b200 import synth
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        db = synth.generate(4, scale=0.01)
        off_all, items_all = db.offsets.astype(np.int64), db.items.astype(np.int32)
        off, items = shard_csr(off_all, items_all, rank, world)
        # whole-database id range and F1 from the shards (MAX, then SUM)
        mx = torch.tensor([int(items.max()) if items.size else -1], dtype=torch.int64)
        dist.all_reduce(mx, op=dist.ReduceOp.MAX)
        f1 = torch.from_numpy(np.bincount(items, minlength=int(mx) + 1).astype(np.int32))
        dist.all_reduce(f1, op=dist.ReduceOp.SUM)
        n_all = torch.tensor([off.shape[0] - 1], dtype=torch.int64)
        dist.all_reduce(n_all, op=dist.ReduceOp.SUM)
        f1 = f1.numpy()
        assert int(n_all) == off_all.shape[0] - 1
        np.testing.assert_array_equal(f1, np.bincount(items_all, minlength=f1.shape[0]))
        min_count = int(np.ceil(int(n_all) * 0.004))
        surv = [i for i in range(1, f1.shape[0]) if f1[i] >= min_count]
        dense_of = np.full(f1.shape[0], -1, np.int64)
        dense_of[surv] = np.arange(len(surv))
        d = len(surv)
        rng = np.random.default_rng(3)
        lists = [sorted(rng.choice(d, size=int(rng.integers(1, 4)), replace=False).tolist()) for _ in range(64)]
        part, part_nfreq = oracle.count_wave(_bitmap(off, items, dense_of, d), lists, d, min_count)
        summed = torch.from_numpy(part.copy())
        dist.all_reduce(summed, op=dist.ReduceOp.SUM)
        whole, whole_nfreq = oracle.count_wave(_bitmap(off_all, items_all, dense_of, d), lists, d, min_count)
        np.testing.assert_array_equal(summed.numpy(), whole)
        np.testing.assert_array_equal((summed.numpy() >= min_count).sum(axis=1), whole_nfreq)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), np.array([int(part_nfreq.sum()), int(whole_nfreq.sum())]))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_partial_counts_exactly(tmp_path, oracle_mod):
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True,
                       start_method="spawn")
    res = [np.load(tmp_path / f"r{r}.npy") for r in range(world)]
    assert res[0][1] == res[1][1]
    # thresholding a shard's partial counts alone would lose frequent extensions
    assert all(r[0] < r[1] for r in res)
